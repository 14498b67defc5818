// skg_api.cu -- the C ABI (include/skirt_b200.h): contexts, scene upload, phase launches,
// tallies, the bit-exact path harness and the grid builders.
#include "skg_scene.cuh"
#include "skg_internal.h"
#include "skg_tree.h"
#include "skg_wave.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

using namespace skg;

namespace {

// Device allocations of one owner.  With a stream set they are stream-ordered (cudaMallocAsync /
// cudaFreeAsync on that stream): releasing a context then does not synchronise the device, which
// a plain cudaFree does -- a serving loop frees retired contexts while other simulations run.  The
// owner synchronises the stream before another stream uses the memory.
struct Allocs {
    std::vector<void*> ptrs;
    size_t bytes = 0;
    cudaStream_t stream = nullptr;
    ~Allocs() { release(); }
    void release() {
        for (void* p : ptrs) {
            if (stream) cudaFreeAsync(p, stream); else cudaFree(p);
        }
        ptrs.clear(); bytes = 0;
    }
    template<typename T> T* alloc(size_t n) {
        if (n == 0) n = 1;
        void* p = nullptr;
        const cudaError_t e = stream ? cudaMallocAsync(&p, n * sizeof(T), stream) : cudaMalloc(&p, n * sizeof(T));
        if (e != cudaSuccess) { cudaGetLastError(); return nullptr; }
        ptrs.push_back(p); bytes += n * sizeof(T);
        return (T*)p;
    }
};

struct Failure { int code; std::string msg; };
// A failed call throws its status: SKG_ERR_OOM for an allocation the device cannot satisfy (a
// non-sticky error, cleared here so that the context stays usable), SKG_ERR_CUDA otherwise.
#define CK(expr) do { cudaError_t e_ = (expr); if (e_ != cudaSuccess) {                          \
        if (e_ == cudaErrorMemoryAllocation) cudaGetLastError();                                  \
        throw Failure{e_ == cudaErrorMemoryAllocation ? SKG_ERR_OOM : SKG_ERR_CUDA,                \
                      std::string(#expr) + ": " + cudaGetErrorString(e_)}; } } while (0)
#define REQUIRE(cond, msg) do { if (!(cond)) throw Failure{SKG_ERR_INVALID, msg}; } while (0)

template<typename T> T* upload(Allocs& A, const T* h, size_t n, cudaStream_t s) {
    T* d = A.alloc<T>(n);
    if (!d) throw Failure{SKG_ERR_OOM, "device allocation failed"};
    if (h && n) CK(cudaMemcpyAsync(d, h, n * sizeof(T), cudaMemcpyHostToDevice, s));
    return d;
}
template<typename T> T* zeros(Allocs& A, size_t n, cudaStream_t s) {
    T* d = A.alloc<T>(n);
    if (!d) throw Failure{SKG_ERR_OOM, "device allocation failed"};
    CK(cudaMemsetAsync(d, 0, std::max<size_t>(n, 1) * sizeof(T), s));
    return d;
}

// cubic spline kernel cumulative mass table (CubicSplineSmoothingKernel.cpp:22-38)
std::vector<double> cubic_spline_table() {
    const int Nu = 400;
    std::vector<double> X(Nu + 1);
    for (int k = 0; k <= Nu; k++) {
        double u = k * (1.0 / Nu), u2 = u * u, u3 = u * u2;
        X[k] = (u < 0.5) ? u3 * (32.0 / 3.0 - 192.0 / 5.0 * u2 + 32.0 * u3)
                         : -1.0 / 15.0 - 64.0 * u3 * (-1.0 / 3.0 + 0.75 * u - 0.6 * u2 + u3 / 6.0);
    }
    return X;
}

// Builds the device form of a geometry (tables uploaded into A).
DevGeometry make_geometry(Allocs& A, const skg_geometry& g, cudaStream_t s) {
    DevGeometry G;
    std::memset(&G, 0, sizeof(G));
    G.type = g.type;
    for (int i = 0; i < 6; i++) G.p[i] = g.p[i];
    if (g.type == SKG_GEOM_EXPDISK) {
        // ExpDiskGeometry::setupSelfBefore (ExpDiskGeometry.cpp:24-40)
        G.hR = g.p[0]; G.hz = g.p[1]; G.Rmax = g.p[2]; G.zmax = g.p[3]; G.Rmin = g.p[4];
        REQUIRE(G.hR > 0 && G.hz > 0, "exponential disk scale lengths must be positive");
        double intz = (G.zmax > 0) ? -2.0 * G.hz * std::expm1(-G.zmax / G.hz) : 2.0 * G.hz;
        double tmin = (G.Rmin > 0) ? std::exp(-G.Rmin / G.hR) * (1.0 + G.Rmin / G.hR) : 1.0;
        double tmax = (G.Rmax > 0) ? std::exp(-G.Rmax / G.hR) * (1.0 + G.Rmax / G.hR) : 0.0;
        G.rho0 = 1.0 / (G.hR * G.hR * (tmin - tmax) * 2.0 * M_PI * intz);
    } else if (g.type == SKG_GEOM_SERSIC) {
        REQUIRE(g.p[0] > 0.5 && g.p[0] <= 10 && g.p[1] > 0, "Sersic index must be in (0.5,10] and radius positive");
        std::vector<double> sv(101), Sv(101), Mv(101);
        sersic_table(g.p[0], sv.data(), Sv.data(), Mv.data());
        G.sv = upload(A, sv.data(), 101, s); G.Sv = upload(A, Sv.data(), 101, s); G.Mv = upload(A, Mv.data(), 101, s);
        G.reff = g.p[1]; G.srho0 = 1.0 / (G.reff * G.reff * G.reff);
    } else if (g.type == SKG_GEOM_PLUMMER) {
        REQUIRE(g.p[0] > 0, "Plummer scale radius must be positive");
    } else {
        REQUIRE(g.type == SKG_GEOM_POINT, "unknown geometry type");
    }
    if (g.clump_count > 0) {
        REQUIRE(g.clump_pos != nullptr, "clumpy geometry needs clump positions");
        REQUIRE(g.clump_fraction >= 0 && g.clump_fraction <= 1 && g.clump_radius > 0, "invalid clump parameters");
        G.f = g.clump_fraction; G.N = g.clump_count; G.h = g.clump_radius; G.cutoff = g.clump_cutoff;
        G.kernel = g.clump_kernel;
        std::vector<int> idx(G.N);
        for (int i = 0; i < G.N; i++) idx[i] = i;
        std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return g.clump_pos[3 * a] < g.clump_pos[3 * b]; });
        std::vector<double> cl(3 * (size_t)G.N);
        for (int i = 0; i < G.N; i++) for (int c = 0; c < 3; c++) cl[3 * i + c] = g.clump_pos[3 * idx[i] + c];
        G.clumps = upload(A, cl.data(), cl.size(), s);
        std::vector<double> kx = cubic_spline_table();
        G.kXv = upload(A, kx.data(), kx.size(), s);
    }
    return G;
}

double grid_diag(const skg_grid& g) {
    double dx = g.xmax - g.xmin, dy = g.ymax - g.ymin, dz = g.zmax - g.zmin;
    return std::sqrt(dx * dx + dy * dy + dz * dz);
}

// the FP32 Cartesian walk computes the walls of evenly spaced grids (1) or loads them from the
// plane tables for every grid (0): traversal pass of a 10^7-packet phase of the oligochromatic disk
// 61.6 against 64.1 ms, a batch of 24 fit variants 571 against 605 ms
#ifndef SKG_CART_UNIFORM
#define SKG_CART_UNIFORM 1
#endif

// Uploads a grid into both precisions.
DevGrid make_grid(Allocs& A, const skg_grid& g, cudaStream_t s) {
    DevGrid G;
    std::memset(&G, 0, sizeof(G));
    G.type = g.type;
    G.xmin = g.xmin; G.ymin = g.ymin; G.zmin = g.zmin; G.xmax = g.xmax; G.ymax = g.ymax; G.zmax = g.zmax;
    REQUIRE(g.xmax > g.xmin && g.ymax > g.ymin && g.zmax > g.zmin, "grid extent is empty");
    double diag = grid_diag(g);
    G.eps = 1e-12 * diag;
    double amax = std::max({std::fabs(g.xmin), std::fabs(g.xmax), std::fabs(g.ymin), std::fabs(g.ymax),
                            std::fabs(g.zmin), std::fabs(g.zmax)});
    // FP32 nudge: four units in the last place of the largest coordinate
    G.epsf = (float)std::max(4.0 * amax * std::ldexp(1.0, -23), 1e-12 * diag);
    G.max_steps = 1 << 20;
    if (g.type == SKG_GRID_CARTESIAN) {
        REQUIRE(g.nx > 0 && g.ny > 0 && g.nz > 0 && g.xv && g.yv && g.zv, "Cartesian grid needs planes");
        REQUIRE((int64_t)g.nx * g.ny * g.nz < (1ll << 31), "too many Cartesian cells");
        G.nx = g.nx; G.ny = g.ny; G.nz = g.nz;
        G.xv = upload(A, g.xv, g.nx + 1, s); G.yv = upload(A, g.yv, g.ny + 1, s); G.zv = upload(A, g.zv, g.nz + 1, s);
        std::vector<float> f;
        f.assign(g.xv, g.xv + g.nx + 1); G.xvf = upload(A, f.data(), f.size(), s);
        f.assign(g.yv, g.yv + g.ny + 1); G.yvf = upload(A, f.data(), f.size(), s);
        f.assign(g.zv, g.zv + g.nz + 1); G.zvf = upload(A, f.data(), f.size(), s);
        G.ncells = g.nx * g.ny * g.nz;
        // evenly spaced planes (to 1e-9 of the spacing) on all three axes: the FP32 walk computes
        // its walls
        auto even = [](const double* v, int n, float& org, float& h) {
            const double step = (v[n] - v[0]) / n;
            for (int q = 0; q <= n; q++)
                if (std::fabs(v[q] - (v[0] + q * step)) > 1e-9 * std::fabs(step)) return false;
            org = (float)v[0]; h = (float)step;
            return step > 0;
        };
        G.cart_uniform = SKG_CART_UNIFORM && even(g.xv, g.nx, G.corg[0], G.cstep[0]) &&
                         even(g.yv, g.ny, G.corg[1], G.cstep[1]) && even(g.zv, g.nz, G.corg[2], G.cstep[2]);
    } else if (g.type == SKG_GRID_OCTREE || g.type == SKG_GRID_BINTREE) {
        int n = g.nnodes;
        REQUIRE(n > 0 && g.node_box && g.node_child && g.node_father && g.node_cell && g.node_dir, "tree grid needs node arrays");
        G.nnodes = n;
        G.node_box = upload(A, g.node_box, 6 * (size_t)n, s);
        G.node_child = upload(A, g.node_child, n, s);
        G.node_father = upload(A, g.node_father, n, s);
        G.node_cell = upload(A, g.node_cell, n, s);
        G.node_dir = upload(A, (const signed char*)g.node_dir, n, s);
        std::vector<float4> nf(2 * (size_t)n);
        int nc = 0;
        for (int l = 0; l < n; l++) {
            const double* b = g.node_box + 6 * (size_t)l;
            int ch = g.node_child[l], ce = g.node_cell[l];
            float4 a, c;
            a.x = (float)b[0]; a.y = (float)b[1]; a.z = (float)b[2]; std::memcpy(&a.w, &ch, 4);
            c.x = (float)b[3]; c.y = (float)b[4]; c.z = (float)b[5]; std::memcpy(&c.w, &ce, 4);
            nf[2 * l] = a; nf[2 * l + 1] = c;
            if (ce >= 0) nc++;
        }
        G.nodef = upload(A, nf.data(), nf.size(), s);
        std::vector<int> cn(nc);
        for (int l = 0; l < n; l++) if (g.node_cell[l] >= 0) {
            REQUIRE(g.node_cell[l] < nc, "leaf cell number out of range");
            cn[g.node_cell[l]] = l;
        }
        G.cell_node = upload(A, cn.data(), cn.size(), s);
        G.ncells = nc;
        G.search = g.search_method;
        if (g.search_method == SKG_SEARCH_NEIGHBOR) {
            REQUIRE(g.nbr_offsets && g.nbr_ids, "neighbour search needs neighbour lists");
            int64_t tot = g.nbr_offsets[6 * (size_t)n];
            REQUIRE(tot < (1ll << 31), "too many neighbour entries");
            std::vector<int> off(6 * (size_t)n + 1);
            for (size_t q = 0; q <= 6 * (size_t)n; q++) off[q] = (int)g.nbr_offsets[q];
            G.nbroff = upload(A, off.data(), off.size(), s);
            G.nbr = upload(A, g.nbr_ids, (size_t)tot, s);
        }
        // rope-linked tree for the FP32 walk
        {
            RopeTree rt;
            // SKG_TREE_RECORDS=rope keeps the 64-byte leaf records for trees that fit the lattice
            const char* rec = std::getenv("SKG_TREE_RECORDS");
            build_rope_tree(g, rt, !(rec && std::strcmp(rec, "rope") == 0));
            if (rt.lattice) {
                G.prec = upload(A, rt.prec.data(), rt.prec.size(), s);
                G.lattice = 1;
                for (int a = 0; a < 3; a++) { G.lorg[a] = rt.lorg[a]; G.lunit[a] = rt.lunit[a]; }
            } else {
                G.lrec = upload(A, rt.lrec.data(), rt.lrec.size(), s);
            }
            G.irec = upload(A, rt.irec.data(), std::max<size_t>(rt.irec.size(), 1), s);
            G.cell_leaf = upload(A, rt.cell_leaf.data(), rt.cell_leaf.size(), s);
            G.root_ref = rt.root_ref;
        }
        REQUIRE(g.search_method != SKG_SEARCH_BOOKKEEPING || g.type == SKG_GRID_OCTREE,
                "the bookkeeping search method requires an octree");
    } else if (g.type == SKG_GRID_VORONOI) {
        int n = g.nsites;
        REQUIRE(n > 0 && g.sites && g.vnbr_offsets && g.vnbr_ids && g.nb > 0 && g.block_offsets && g.block_ids,
                "Voronoi grid needs sites, neighbour lists and block lists");
        G.nsites = n; G.ncells = n;
        G.site = upload(A, g.sites, 3 * (size_t)n, s);
        std::vector<float4> sf(n);
        for (int m = 0; m < n; m++) sf[m] = make_float4((float)g.sites[3 * m], (float)g.sites[3 * m + 1], (float)g.sites[3 * m + 2], 0.f);
        G.sitef = upload(A, sf.data(), sf.size(), s);
        int64_t tot = g.vnbr_offsets[n];
        REQUIRE(tot < (1ll << 31), "too many Voronoi neighbour entries");
        std::vector<int> off(n + 1);
        for (int m = 0; m <= n; m++) off[m] = (int)g.vnbr_offsets[m];
        G.vnoff = upload(A, off.data(), off.size(), s);
        G.vnbr = upload(A, g.vnbr_ids, (size_t)tot, s);
        // FP32 bisector planes: n = p_i - p_r, w = n . (p_i + p_r)/2 (computed in FP64, stored FP32);
        // walls -1..-6 as axis planes with outward normals
        std::vector<float4> pl((size_t)tot);
        for (int m = 0; m < n; m++) {
            const double* pr = g.sites + 3 * (size_t)m;
            for (int64_t q = g.vnbr_offsets[m]; q < g.vnbr_offsets[m + 1]; q++) {
                int mi = g.vnbr_ids[q];
                double nx, ny, nz, w;
                if (mi >= 0) {
                    REQUIRE(mi < n, "Voronoi neighbour id out of range");
                    const double* pi = g.sites + 3 * (size_t)mi;
                    nx = pi[0] - pr[0]; ny = pi[1] - pr[1]; nz = pi[2] - pr[2];
                    // unit normal: n.p with unnormalised n (~1e19 m x 1e20 m) overflows FP32
                    double inv = 1.0 / std::sqrt(nx * nx + ny * ny + nz * nz);
                    nx *= inv; ny *= inv; nz *= inv;
                    w = nx * 0.5 * (pi[0] + pr[0]) + ny * 0.5 * (pi[1] + pr[1]) + nz * 0.5 * (pi[2] + pr[2]);
                } else {
                    nx = ny = nz = 0;
                    switch (mi) {
                        case -1: nx = -1; w = -g.xmin; break;
                        case -2: nx = 1;  w = g.xmax; break;
                        case -3: ny = -1; w = -g.ymin; break;
                        case -4: ny = 1;  w = g.ymax; break;
                        case -5: nz = -1; w = -g.zmin; break;
                        case -6: nz = 1;  w = g.zmax; break;
                        default: throw Failure{SKG_ERR_INVALID, "invalid Voronoi wall id"};
                    }
                }
                pl[q] = make_float4((float)nx, (float)ny, (float)nz, (float)w);
            }
        }
        G.vplane = upload(A, pl.data(), pl.size(), s);
        // per entry the neighbour with its own entry range, so that the FP32 walk reaches the next
        // cell's planes with one load
        std::vector<int4> nx4((size_t)tot);
        for (int64_t q = 0; q < tot; q++) {
            int mi = g.vnbr_ids[q];
            nx4[q] = (mi >= 0) ? make_int4(mi, off[mi], off[mi + 1], 0) : make_int4(mi, 0, 0, 0);
        }
        G.vnext = upload(A, nx4.data(), nx4.size(), s);
        G.nb = g.nb;
        size_t nb3 = (size_t)g.nb * g.nb * g.nb;
        int64_t btot = g.block_offsets[nb3];
        REQUIRE(btot < (1ll << 31), "too many block list entries");
        std::vector<int> boff(nb3 + 1);
        for (size_t b = 0; b <= nb3; b++) boff[b] = (int)g.block_offsets[b];
        G.boff = upload(A, boff.data(), boff.size(), s);
        G.bids = upload(A, g.block_ids, (size_t)btot, s);
        if (g.cell_bbox) G.vbbox = upload(A, g.cell_bbox, 6 * (size_t)n, s);
        else {
            std::vector<double> bb(6 * (size_t)n);
            for (int m = 0; m < n; m++) { bb[6*m] = g.xmin; bb[6*m+1] = g.ymin; bb[6*m+2] = g.zmin; bb[6*m+3] = g.xmax; bb[6*m+4] = g.ymax; bb[6*m+5] = g.zmax; }
            G.vbbox = upload(A, bb.data(), bb.size(), s);
        }
        if (g.cell_volume) G.vvol = upload(A, g.cell_volume, n, s);
        else G.vvol = zeros<double>(A, n, s);
    } else {
        throw Failure{SKG_ERR_INVALID, "unknown grid type"};
    }
    return G;
}

double planck_B(double lambda, double T) {   // PlanckFunction.cpp:24-33
    const double h = 6.62606957e-34, c = 2.99792458e8, k = 1.3806488e-23;
    double x = h * c / (lambda * k * T);
    return 2.0 * h * c * c / std::pow(lambda, 5) / (std::exp(x) - 1.0);
}

}  // namespace

// Device tables of one launch (header, work items, scene slots, wavelength list) and its
// counters; filled from host memory before each launch.
struct Staging {
    BatchHeader* hdr = nullptr;
    WorkItem* items = nullptr;
    DevGrid* grids = nullptr;
    const DevScene** scenes = nullptr;
    int* ells = nullptr;
    unsigned long long* work = nullptr;
    unsigned* err = nullptr;
    unsigned long long* counters = nullptr;
    int max_items = 0, max_slots = 0, max_ells = 0;
    void alloc(Allocs& A, int items, int slots, int nells) {
        max_items = items; max_slots = slots; max_ells = nells;
        hdr = A.alloc<BatchHeader>(1); this->items = A.alloc<WorkItem>(items); grids = A.alloc<DevGrid>(slots);
        scenes = (const DevScene**)A.alloc<void*>(slots); ells = A.alloc<int>(nells);
        work = A.alloc<unsigned long long>(1); err = A.alloc<unsigned>(1); counters = A.alloc<unsigned long long>(10);
        if (!hdr || !this->items || !grids || !scenes || !ells || !work || !err || !counters)
            throw Failure{SKG_ERR_OOM, "device allocation failed"};
    }
    RunParams params(int max_scatt, int refill = 0) const {
        RunParams P;
        std::memset(&P, 0, sizeof(P));
        P.hdr = hdr; P.items = items; P.grids = grids; P.scenes = scenes; P.ells = ells;
        P.max_scatt = max_scatt; P.refill = refill; P.work = work; P.err = err; P.counters = counters;
        return P;
    }
};

struct skg_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    float last_ms = 0;
    Allocs A;
    DevGrid grid;
    DevScene hs;
    DevScene* ds = nullptr;
    int nlambda = 0, ncomp = 0;
    int64_t ncells = 0;
    std::vector<int64_t> cube_len, sed_len;
    unsigned long long* counters = nullptr;   // = own.counters
    unsigned* err = nullptr;                  // = own.err (the phases' error word)
    // The path harness (skg_trace_paths, skg_optical_depth, skg_trace_paths_noalloc) flags its
    // errors in a word of its own, so that a harness call never clears a finished phase's flags
    // before skg_sync has reported them.  hev marks the end of the last no-alloc call on the
    // caller's stream; skg_sync waits for it before it reads herr.
    unsigned* herr = nullptr;
    cudaEvent_t hev = nullptr;
    bool hev_pending = false;
    Staging own;                              // tables of this context's own launches
    WaveRunner waves;                         // packet pool and job lists of this context's phases
    uint64_t wave_count = 0;                  // waves since the last tally reset
    std::vector<double> lambda, dlambda;
    // dust emission
    int nT = 0;
    double *Tv = nullptr, *planckabs = nullptr, *labsbol = nullptr, *spectra = nullptr, *temperature = nullptr;
    double *emit_Lv = nullptr, *emit_cdf = nullptr, *emit_Ltot = nullptr, *sumbuf = nullptr;
    void* scan_scratch = nullptr; size_t scan_bytes = 0;
    std::string error;
};

static int fail(skg_ctx* ctx, const Failure& f) {
    set_error(f.msg);
    if (ctx) ctx->error = f.msg;
    return f.code;
}

// Completes the context's running phase: waits for its enqueued waves and adds waves until no
// packet is left (the reads, resets and the next phase need the finished tallies).
static int settle(skg_ctx* ctx, int timeout_ms) {
    if (!ctx->waves.pending()) return SKG_OK;
    cudaSetDevice(ctx->device);
    bool timed_out = false;
    cudaError_t e = ctx->waves.finish(timeout_ms, ctx->ev1, &timed_out);
    if (e != cudaSuccess) { cudaGetLastError(); return fail(ctx, Failure{SKG_ERR_CUDA, cudaGetErrorString(e)}); }
    if (timed_out) return fail(ctx, Failure{SKG_ERR_TIMEOUT, "timed out waiting for the device"});
    ctx->wave_count += ctx->waves.waves();
    return SKG_OK;
}

extern "C" {

int skg_version(void) { return SKG_ABI_VERSION; }

const char* skg_last_error(const skg_ctx* ctx) {
    if (ctx && !ctx->error.empty()) return ctx->error.c_str();
    return get_error();
}

int skg_device_count(int* count) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) { cudaGetLastError(); *count = 0; set_error(cudaGetErrorString(e)); return SKG_ERR_NO_DEVICE; }
    *count = n;
    return SKG_OK;
}

int skg_chunk_params(double packages, int nthreads, int nprocs, int nlambda,
                     uint64_t* nchunks, uint64_t* chunksize, uint64_t* npp) {
    chunk_params(packages, nthreads, nprocs, nlambda, *nchunks, *chunksize, *npp);
    return SKG_OK;
}

int skg_ctx_create(const skg_scene* sc, int device, skg_ctx** out) {
    *out = nullptr;
    skg_ctx* ctx = new skg_ctx();
    try {
        REQUIRE(sc != nullptr, "scene is null");
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { cudaGetLastError(); throw Failure{SKG_ERR_NO_DEVICE, "no CUDA device"}; }
        REQUIRE(device >= 0 && device < ndev, "device index out of range");
        ctx->device = device;
        CK(cudaSetDevice(device));
        CK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
        CK(cudaEventCreate(&ctx->ev0)); CK(cudaEventCreate(&ctx->ev1));
        ctx->waves.timing = true;
        cudaStream_t s = ctx->stream;
        Allocs& A = ctx->A;
        A.stream = s;                      // stream-ordered; the stream is synchronised below

        REQUIRE(sc->nlambda > 0 && sc->lambda && sc->dlambda, "wavelength grid is empty");
        REQUIRE(sc->ncomp >= 0 && sc->ncomp <= MAX_COMP, "at most 4 dust components");
        REQUIRE(sc->nstellar >= 1 && sc->nstellar <= MAX_STELLAR, "1..8 stellar components");
        REQUIRE(sc->ninstr >= 0 && sc->ninstr <= MAX_INSTR, "at most 16 instruments");
        REQUIRE(sc->scatt_bias >= 0 && sc->scatt_bias <= 1, "The scattering bias should be between 0 and 1");
        REQUIRE(sc->min_weight_reduction == 0 || sc->min_weight_reduction >= 1e3,
                "The minimum weight reduction factor should be larger than 1000");
        REQUIRE(sc->min_scatt_events >= 0 && sc->min_scatt_events <= 1000, "minScattEvents out of range");
        const int nl = sc->nlambda;
        ctx->nlambda = nl; ctx->ncomp = sc->ncomp;
        ctx->lambda.assign(sc->lambda, sc->lambda + nl);
        ctx->dlambda.assign(sc->dlambda, sc->dlambda + nl);

        DevScene& H = ctx->hs;
        std::memset(&H, 0, sizeof(H));
        ctx->grid = make_grid(A, sc->grid, s);
        ctx->ncells = ctx->grid.ncells;
        const int64_t nc = ctx->ncells;
        H.ncells = (int)nc;
        H.nlambda = nl;
        H.lambda = upload(A, sc->lambda, nl, s);
        H.dlambda = upload(A, sc->dlambda, nl, s);

        // dust mixes (SimpleOligoDustMix.cpp:38-45: kappa_abs = kappa_ext(1-a), kappa_sca = kappa_ext a)
        H.ncomp = sc->ncomp;
        if (sc->ncomp > 0) {
            std::vector<double> ke(sc->ncomp * nl), ks(sc->ncomp * nl), al(sc->ncomp * nl), gg(sc->ncomp * nl);
            std::vector<DevGeometry> dg(sc->ncomp);
            std::vector<double> norms(sc->ncomp);
            for (int h = 0; h < sc->ncomp; h++) {
                const skg_dust_comp& d = sc->dust[h];
                REQUIRE(d.kappaext && d.albedo && d.asymmpar, "dust mix tables missing");
                for (int l = 0; l < nl; l++) {
                    ke[h * nl + l] = d.kappaext[l]; al[h * nl + l] = d.albedo[l]; gg[h * nl + l] = d.asymmpar[l];
                    ks[h * nl + l] = d.kappaext[l] * d.albedo[l];
                    REQUIRE(d.kappaext[l] >= 0 && d.albedo[l] >= 0 && d.albedo[l] <= 1 && std::fabs(d.asymmpar[l]) < 1,
                            "invalid dust mix values");
                }
                if (!sc->rho) dg[h] = make_geometry(A, d.geometry, s);
                norms[h] = d.norm;
            }
            H.kext = upload(A, ke.data(), ke.size(), s);
            H.ksca = upload(A, ks.data(), ks.size(), s);
            H.albedo = upload(A, al.data(), al.size(), s);
            H.asym = upload(A, gg.data(), gg.size(), s);
            double* rho;
            if (sc->rho) {
                for (int64_t i = 0; i < nc * sc->ncomp; i++)
                    REQUIRE(sc->rho[i] >= 0 && std::isfinite(sc->rho[i]), "cell densities must be finite and non-negative");
                rho = upload(A, sc->rho, (size_t)(nc * sc->ncomp), s);
            } else {
                // DustSystem::setSampleDensityBody on the device
                rho = A.alloc<double>(nc * sc->ncomp);
                if (!rho) throw Failure{SKG_ERR_OOM, "device allocation failed"};
                DevGeometry* dgd = upload(A, dg.data(), dg.size(), s);
                double* nd = upload(A, norms.data(), norms.size(), s);
                CK(launch_sample_density(ctx->grid, nullptr, dgd, nd, sc->ncomp,
                                         sc->density_samples > 0 ? sc->density_samples : 100, 0x5EED0001ull, rho, s));
            }
            H.rho = rho;
            float* rf = A.alloc<float>(nc * sc->ncomp);
            if (!rf) throw Failure{SKG_ERR_OOM, "device allocation failed"};
            {
                std::vector<double> hr(nc * sc->ncomp);
                CK(cudaMemcpyAsync(hr.data(), rho, hr.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
                CK(cudaStreamSynchronize(s));
                std::vector<float> hf(hr.begin(), hr.end());
                CK(cudaMemcpyAsync(rf, hf.data(), hf.size() * sizeof(float), cudaMemcpyHostToDevice, s));
                CK(cudaStreamSynchronize(s));
            }
            H.rhof = rf;
            if (sc->ncomp == 1 && (ctx->grid.lrec || ctx->grid.prec)) CK(launch_embed_density(ctx->grid, rf, s));
        }

        // stellar system (StellarSystem.cpp:35-52)
        H.nstellar = sc->nstellar;
        std::vector<double> starL(sc->nstellar * nl), Lv(nl, 0.0), Xvv((size_t)nl * (sc->nstellar + 1), 0.0);
        for (int h = 0; h < sc->nstellar; h++) {
            REQUIRE(sc->stellar[h].luminosity, "stellar luminosities missing");
            H.stellar[h] = make_geometry(A, sc->stellar[h].geometry, s);
            for (int l = 0; l < nl; l++) {
                starL[h * nl + l] = sc->stellar[h].luminosity[l];
                REQUIRE(starL[h * nl + l] >= 0, "stellar luminosity must be non-negative");
            }
        }
        for (int l = 0; l < nl; l++) {
            double* X = &Xvv[(size_t)l * (sc->nstellar + 1)];
            for (int h = 0; h < sc->nstellar; h++) { Lv[l] += starL[h * nl + l]; X[h + 1] = X[h] + starL[h * nl + l]; }
            double t = X[sc->nstellar];
            for (int h = 0; h <= sc->nstellar; h++) X[h] = (t > 0) ? X[h] / t : 0.0;
        }
        H.starL = upload(A, starL.data(), starL.size(), s);
        H.Lv = upload(A, Lv.data(), Lv.size(), s);
        H.Xvv = upload(A, Xvv.data(), Xvv.size(), s);
        H.emission_bias = sc->emission_bias;

        // instruments (DistantInstrument.cpp:27-50, SingleFrameInstrument.cpp:26-42)
        H.ninstr = sc->ninstr;
        ctx->cube_len.assign(sc->ninstr, 0); ctx->sed_len.assign(sc->ninstr, 0);
        for (int i = 0; i < sc->ninstr; i++) {
            const skg_instrument& in = sc->instr[i];
            DevInstr& I = H.instr[i];
            std::memset(&I, 0, sizeof(I));
            REQUIRE(in.distance > 0, "Distance was not set");
            I.type = in.type;
            I.costheta = std::cos(in.inclination); I.sintheta = std::sin(in.inclination);
            I.cosphi = std::cos(in.azimuth); I.sinphi = std::sin(in.azimuth);
            I.cospa = std::cos(in.position_angle); I.sinpa = std::sin(in.position_angle);
            // Direction(theta, phi) (Direction.cpp:12-38)
            double th = in.inclination, ph = in.azimuth;
            if (th <= 1e-8) { I.kx = 0; I.ky = 0; I.kz = 1; }
            else if (th >= M_PI - 1e-8) { I.kx = 0; I.ky = 0; I.kz = -1; }
            else { I.kx = std::sin(th) * std::cos(ph); I.ky = std::sin(th) * std::sin(ph); I.kz = std::cos(th); }
            I.ncomp = 1;
            if (in.type == SKG_INSTR_FRAME && in.stellar_comps) I.ncomp = 1 + std::max(sc->nstellar, 0);
            if (in.type == SKG_INSTR_FULL) { REQUIRE(in.nscatt_levels >= 0, "scattering levels must be >= 0"); I.nscatt_levels = in.nscatt_levels; I.ncomp = SKG_FULL_NBASE + in.nscatt_levels; }
            if (in.type != SKG_INSTR_SED) {
                REQUIRE(in.type == SKG_INSTR_FRAME || in.type == SKG_INSTR_SIMPLE || in.type == SKG_INSTR_FULL, "unknown instrument type");
                REQUIRE(in.nxp > 0 && in.nyp > 0, "Number of pixels was not set");
                REQUIRE(in.fovx > 0 && in.fovy > 0, "Field of view was not set");
                I.nxp = in.nxp; I.nyp = in.nyp;
                I.xpmin = in.xc - 0.5 * in.fovx; I.xpsiz = in.fovx / in.nxp;
                I.ypmin = in.yc - 0.5 * in.fovy; I.ypsiz = in.fovy / in.nyp;
                ctx->cube_len[i] = (int64_t)I.ncomp * nl * in.nxp * in.nyp;
                I.cube = zeros<double>(A, ctx->cube_len[i], s);
            }
            ctx->sed_len[i] = (int64_t)I.ncomp * nl;
            I.sed = zeros<double>(A, ctx->sed_len[i], s);
            H.sed_base[i] = H.sed_bins;
            H.sed_bins += (int)ctx->sed_len[i];
        }
        // direction groups: instruments with the same observer direction share one peel-off traversal
        {
            int ng = 0, pos = 0;
            std::vector<int> assigned(sc->ninstr, -1);
            for (int i = 0; i < sc->ninstr; i++) {
                if (assigned[i] >= 0) continue;
                H.group_start[ng] = pos;
                H.gkx[ng] = H.instr[i].kx; H.gky[ng] = H.instr[i].ky; H.gkz[ng] = H.instr[i].kz;
                bool frame_only = true;
                for (int j = i; j < sc->ninstr; j++) {
                    if (assigned[j] >= 0) continue;
                    if (j == i || (H.instr[j].kx == H.instr[i].kx && H.instr[j].ky == H.instr[i].ky && H.instr[j].kz == H.instr[i].kz)) {
                        assigned[j] = ng; H.group_instr[pos++] = j;
                        if (H.instr[j].type != SKG_INSTR_FRAME) frame_only = false;
                    }
                }
                H.group_frame_only[ng] = frame_only;
                ng++;
            }
            H.group_start[ng] = pos;
            H.ngroups = ng;
        }

        H.min_weight_reduction = sc->min_weight_reduction > 0 ? sc->min_weight_reduction : 1e4;
        H.min_scatt_events = sc->min_scatt_events;
        H.xi = sc->scatt_bias;
        H.store_abs = (sc->store_absorption || sc->dust_emission) ? 1 : 0;
        if (sc->ncomp > 0 && (sc->store_absorption || sc->dust_emission)) {
            H.labs_stel = zeros<double>(A, (size_t)nc * nl, s);
            H.labs_dust = zeros<double>(A, (size_t)nc * nl, s);
        }
        H.dust_emission_bias = sc->dust_emission_bias;

        if (sc->dust_emission && sc->ncomp > 0) {
            REQUIRE(sc->ncomp == 1, "dust emission supports one dust component");
            // temperature grid NR::powgrid(0, 5000, 1000, 500) and Planck-integrated absorption
            // (DustMix.cpp:239-263), with kappa_abs of the mix (the 1/mu factors cancel)
            const int NT = 1000;
            std::vector<double> Tv(NT + 1), pa(NT + 1, 0.0);
            double q = std::pow(500.0, 1. / (NT - 1)), qn = std::pow(q, NT);
            for (int i = 0; i <= NT; ++i) Tv[i] = (1. - std::pow(q, i)) / (1. - qn) * 5000.0;
            for (int p = 1; p <= NT; p++) {
                double acc = 0;
                for (int l = 0; l < nl; l++) {
                    double kabs = sc->dust[0].kappaext[l] * (1.0 - sc->dust[0].albedo[l]);
                    acc += kabs * planck_B(sc->lambda[l], Tv[p]) * sc->dlambda[l];
                }
                pa[p] = acc;
            }
            ctx->nT = NT + 1;
            ctx->Tv = upload(A, Tv.data(), Tv.size(), s);
            ctx->planckabs = upload(A, pa.data(), pa.size(), s);
            ctx->labsbol = zeros<double>(A, nc, s);
            ctx->spectra = zeros<double>(A, (size_t)nc * nl, s);
            ctx->temperature = zeros<double>(A, nc, s);
            ctx->emit_Lv = zeros<double>(A, (size_t)nc * nl, s);
            ctx->emit_cdf = zeros<double>(A, (size_t)(nc + 1) * nl, s);
            ctx->emit_Ltot = zeros<double>(A, nl, s);
            ctx->scan_bytes = emission_scan_scratch_bytes((int)nc);
            ctx->scan_scratch = A.alloc<char>(ctx->scan_bytes);
            H.emit_Lv = ctx->emit_Lv; H.emit_cdf = ctx->emit_cdf; H.emit_Ltot = ctx->emit_Ltot;
        }
        ctx->sumbuf = zeros<double>(A, 2, s);
        ctx->own.alloc(A, 1, 1, nl);
        CK(cudaMemsetAsync(ctx->own.counters, 0, 10 * sizeof(unsigned long long), s));
        CK(cudaMemsetAsync(ctx->own.err, 0, sizeof(unsigned), s));
        ctx->counters = ctx->own.counters;
        ctx->err = ctx->own.err;
        ctx->herr = A.alloc<unsigned>(1);
        if (!ctx->herr) throw Failure{SKG_ERR_OOM, "device allocation failed"};
        CK(cudaMemsetAsync(ctx->herr, 0, sizeof(unsigned), s));
        CK(cudaEventCreateWithFlags(&ctx->hev, cudaEventDisableTiming));
        ctx->ds = upload(A, &H, 1, s);
        CK(cudaStreamSynchronize(s));
        *out = ctx;
        return SKG_OK;
    } catch (const Failure& f) {
        int rc = fail(ctx, f);
        set_error(f.msg);
        if (ctx->stream) cudaStreamSynchronize(ctx->stream);
        ctx->A.release();
        if (ctx->ev0) cudaEventDestroy(ctx->ev0);
        if (ctx->ev1) cudaEventDestroy(ctx->ev1);
        if (ctx->hev) cudaEventDestroy(ctx->hev);
        if (ctx->stream) cudaStreamDestroy(ctx->stream);
        delete ctx;
        return rc;
    }
}

int skg_ctx_destroy(skg_ctx* ctx) {
    if (!ctx) return SKG_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    if (ctx->hev_pending) cudaEventSynchronize(ctx->hev);
    ctx->A.release();
    cudaEventDestroy(ctx->ev0); cudaEventDestroy(ctx->ev1); cudaEventDestroy(ctx->hev);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    return SKG_OK;
}

int skg_ctx_info(const skg_ctx* ctx, int64_t* ncells, int64_t* device_bytes) {
    if (!ctx) return SKG_ERR_INVALID;
    if (ncells) *ncells = ctx->ncells;
    if (device_bytes) *device_bytes = (int64_t)ctx->A.bytes;
    return SKG_OK;
}

int skg_sync(skg_ctx* ctx, int timeout_ms) {
    if (!ctx) return SKG_ERR_INVALID;
    int rc = settle(ctx, timeout_ms);
    if (rc) return rc;
    cudaSetDevice(ctx->device);
    auto t0 = std::chrono::steady_clock::now();
    // the context stream, then the end of the last no-alloc harness call on the caller's stream
    for (int what = 0; what < 2; what++) {
        if (what == 1 && !ctx->hev_pending) break;
        while (true) {
            cudaError_t e = what == 0 ? cudaStreamQuery(ctx->stream) : cudaEventQuery(ctx->hev);
            if (e == cudaSuccess) break;
            if (e != cudaErrorNotReady) { cudaGetLastError(); return fail(ctx, Failure{SKG_ERR_CUDA, cudaGetErrorString(e)}); }
            if (timeout_ms >= 0 && std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count() > timeout_ms)
                return fail(ctx, Failure{SKG_ERR_TIMEOUT, "timed out waiting for the device"});
            std::this_thread::sleep_for(std::chrono::microseconds(200));
        }
    }
    ctx->hev_pending = false;
    unsigned err = 0, herr = 0;
    cudaMemcpy(&err, ctx->err, sizeof(unsigned), cudaMemcpyDeviceToHost);
    cudaMemcpy(&herr, ctx->herr, sizeof(unsigned), cudaMemcpyDeviceToHost);
    if (herr) {
        // a harness failure is reported once
        cudaMemsetAsync(ctx->herr, 0, sizeof(unsigned), ctx->stream);
        cudaStreamSynchronize(ctx->stream);
    }
    if (err & ERR_NAN_TAU) return fail(ctx, Failure{SKG_ERR_NAN_TAU, "The optical depth along the path is not a positive number"});
    if (err & (ERR_STEP_BUDGET | ERR_SCATT_BUDGET)) return fail(ctx, Failure{SKG_ERR_STEP_BUDGET, "a packet exceeded its step or scattering budget"});
    if (err & ERR_CAPACITY) return fail(ctx, Failure{SKG_ERR_CAPACITY, "a packet pool or job list overflowed"});
    if (herr & ERR_CAPACITY) return fail(ctx, Failure{SKG_ERR_CAPACITY, "segment buffer too small"});
    if (herr & ERR_STEP_BUDGET) return fail(ctx, Failure{SKG_ERR_STEP_BUDGET, "a path exceeded the step budget"});
    return SKG_OK;
}

int skg_read_density(skg_ctx* ctx, double* rho) {
    if (!ctx || !rho) return SKG_ERR_INVALID;
    try {
        CK(cudaSetDevice(ctx->device));
        if (ctx->ncomp == 0) return SKG_OK;
        CK(cudaMemcpyAsync(rho, ctx->hs.rho, (size_t)ctx->ncells * ctx->ncomp * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        return SKG_OK;
    } catch (const Failure& f) { return fail(ctx, f); }
}

int skg_trace_paths(skg_ctx* ctx, const double* r, const double* k, int64_t n, int precision,
                    int32_t* cells, double* ds, int64_t* offsets, int64_t capacity) {
    if (!ctx || n < 0 || !offsets) return SKG_ERR_INVALID;
    if (precision != SKG_PREC_FP32 && precision != SKG_PREC_FP64)
        return fail(ctx, Failure{SKG_ERR_INVALID, "skg_trace_paths: unknown precision"});
    int rc = settle(ctx, -1);
    if (rc) return rc;
    try {
        CK(cudaSetDevice(ctx->device));
        cudaStream_t s = ctx->stream;
        Allocs T;
        double* dr = upload(T, r, 3 * (size_t)n, s);
        double* dk = upload(T, k, 3 * (size_t)n, s);
        int64_t* cnt = T.alloc<int64_t>(n + 1);
        if (!cnt) throw Failure{SKG_ERR_OOM, "device allocation failed"};
        CK(cudaMemsetAsync(ctx->herr, 0, sizeof(unsigned), s));
        CK(launch_count_segments(ctx->grid, dr, dk, n, precision, cnt, ctx->herr, s));
        std::vector<int64_t> hc(n);
        if (n) CK(cudaMemcpyAsync(hc.data(), cnt, n * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        offsets[0] = 0;
        for (int64_t i = 0; i < n; i++) offsets[i + 1] = offsets[i] + hc[i];
        int64_t tot = offsets[n];
        if (tot > capacity) throw Failure{SKG_ERR_CAPACITY, "segment buffers too small"};
        int64_t* doff = upload(T, offsets, n + 1, s);
        int32_t* dc = T.alloc<int32_t>(tot);
        double* dd = T.alloc<double>(tot);
        if (!dc || !dd) throw Failure{SKG_ERR_OOM, "device allocation failed"};
        CK(launch_write_segments(ctx->grid, dr, dk, n, precision, doff, dc, dd, ctx->herr, s));
        if (tot) {
            CK(cudaMemcpyAsync(cells, dc, tot * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
            CK(cudaMemcpyAsync(ds, dd, tot * sizeof(double), cudaMemcpyDeviceToHost, s));
        }
        unsigned err = 0;
        CK(cudaMemcpyAsync(&err, ctx->herr, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
        CK(cudaMemsetAsync(ctx->herr, 0, sizeof(unsigned), s));    // reported here, not again by skg_sync
        CK(cudaStreamSynchronize(s));
        if (err & ERR_STEP_BUDGET) throw Failure{SKG_ERR_STEP_BUDGET, "a path exceeded the step budget"};
        if (err & ERR_CAPACITY) throw Failure{SKG_ERR_CAPACITY, "segment count changed between passes"};
        return SKG_OK;
    } catch (const Failure& f) { return fail(ctx, f); }
}

int skg_optical_depth(skg_ctx* ctx, const double* r, const double* k, int64_t n, int ell, int precision, double* tau) {
    if (!ctx || n < 0 || ell < 0 || ell >= ctx->nlambda) return SKG_ERR_INVALID;
    if (precision != SKG_PREC_FP32 && precision != SKG_PREC_FP64)
        return fail(ctx, Failure{SKG_ERR_INVALID, "skg_optical_depth: unknown precision"});
    int rc = settle(ctx, -1);
    if (rc) return rc;
    try {
        CK(cudaSetDevice(ctx->device));
        cudaStream_t s = ctx->stream;
        Allocs T;
        double* dr = upload(T, r, 3 * (size_t)n, s);
        double* dk = upload(T, k, 3 * (size_t)n, s);
        double* dt = T.alloc<double>(n);
        if (n && !dt) throw Failure{SKG_ERR_OOM, "device allocation failed"};
        CK(cudaMemsetAsync(ctx->herr, 0, sizeof(unsigned), s));
        CK(launch_optical_depth(ctx->grid, ctx->ds, dr, dk, n, ell, precision, dt, ctx->herr, s));
        if (n) CK(cudaMemcpyAsync(tau, dt, n * sizeof(double), cudaMemcpyDeviceToHost, s));
        unsigned err = 0;
        CK(cudaMemcpyAsync(&err, ctx->herr, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
        CK(cudaMemsetAsync(ctx->herr, 0, sizeof(unsigned), s));
        CK(cudaStreamSynchronize(s));
        if (err & ERR_STEP_BUDGET) throw Failure{SKG_ERR_STEP_BUDGET, "a path exceeded the step budget"};
        return SKG_OK;
    } catch (const Failure& f) { return fail(ctx, f); }
}

int skg_run_phase(skg_ctx* ctx, int phase, const int32_t* ells, int nell, uint64_t npp, uint64_t first_packet,
                  uint64_t count, uint64_t seed, const skg_run_opts* opts, void* stream) {
    if (!ctx) return SKG_ERR_INVALID;
    int rc = settle(ctx, -1);
    if (rc) return rc;
    try {
        CK(cudaSetDevice(ctx->device));
        REQUIRE(phase >= SKG_PHASE_STELLAR && phase <= SKG_PHASE_DUST_EMISSION, "unknown phase");
        REQUIRE(nell > 0 && ells, "no wavelengths given");
        for (int i = 0; i < nell; i++) REQUIRE(ells[i] >= 0 && ells[i] < ctx->nlambda, "wavelength index out of range");
        REQUIRE(count <= npp || npp == 0, "packet range exceeds the packet count");
        if (phase != SKG_PHASE_STELLAR) REQUIRE(ctx->emit_cdf != nullptr, "dust phases need dust emission enabled");
        REQUIRE(!opts || opts->pool >= 0, "negative packet pool");
        REQUIRE(!opts || opts->precision == SKG_PREC_FP32 || opts->precision == SKG_PREC_FP64, "unknown precision");
        cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
        if (count == 0) return SKG_OK;
        const uint64_t total = (uint64_t)nell * count;
        // packets in flight: 2^21 records (256 MB) by default; a large phase on a grid without
        // re-walk checkpoints (1 KB per record on the Voronoi grid) takes 2^23 (1 GB of records,
        // 4x fewer waves: the 5*10^8-packet octree phase 7.85 s against 8.14 s)
        const bool big = total >= ((uint64_t)1 << 26) && ctx->grid.type != SKG_GRID_VORONOI;
        const size_t pool_max = (opts && opts->pool > 0) ? (size_t)opts->pool : ((size_t)1 << (big ? 23 : 21));
        const size_t npool = (size_t)std::min<uint64_t>(total, pool_max);
        CK(ctx->waves.reserve(npool, ctx->hs.ngroups, ctx->grid.type));
        // one slot, one work item (pageable host sources: the copies are staged before return)
        BatchHeader H = {phase, 1, 1, 0, total};
        WorkItem W;
        std::memset(&W, 0, sizeof(W));
        W.slot = 0; W.nell = nell; W.ell0 = 0; W.npp_total = npp; W.first = first_packet; W.count = count;
        W.seed = seed; W.begin = 0;
        DevGrid g = ctx->grid;
        if (opts && opts->max_steps > 0) g.max_steps = opts->max_steps;
        const DevScene* sp = ctx->ds;
        Staging& T = ctx->own;
        CK(cudaMemcpyAsync(T.hdr, &H, sizeof(H), cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(T.items, &W, sizeof(W), cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(T.grids, &g, sizeof(g), cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(T.scenes, &sp, sizeof(sp), cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(T.ells, ells, nell * sizeof(int), cudaMemcpyHostToDevice, s));
        CK(cudaMemsetAsync(T.work, 0, sizeof(unsigned long long), s));
        CK(cudaMemsetAsync(T.err, 0, sizeof(unsigned), s));
        REQUIRE(!opts || (opts->refill >= 0 && opts->refill <= 32), "refill lanes must be in 0..32");
        RunParams P = T.params((opts && opts->max_scatt > 0) ? opts->max_scatt : 100000, opts ? opts->refill : 0);
        int precision = opts ? opts->precision : SKG_PREC_FP32;
        int blocks = opts ? opts->blocks : 0;
        CK(cudaEventRecord(ctx->ev0, s));
        CK(ctx->waves.begin(P, ctx->grid.type, tree_walk_of(ctx->grid), precision, 1, npool, blocks, s, &g));
        CK(cudaEventRecord(ctx->ev1, s));
        return SKG_OK;
    } catch (const Failure& f) { return fail(ctx, f); }
}

int skg_last_phase_ms(skg_ctx* ctx, float* ms) {
    if (!ctx || !ms) return SKG_ERR_INVALID;
    int rc = settle(ctx, -1);
    if (rc) return rc;
    cudaSetDevice(ctx->device);
    cudaError_t e = cudaEventSynchronize(ctx->ev1);
    if (e != cudaSuccess) { cudaGetLastError(); return fail(ctx, Failure{SKG_ERR_CUDA, cudaGetErrorString(e)}); }
    cudaEventElapsedTime(ms, ctx->ev0, ctx->ev1);
    return SKG_OK;
}

int skg_phase_times(skg_ctx* ctx, float* event_ms, float* traversal_ms, int32_t* waves) {
    if (!ctx) return SKG_ERR_INVALID;
    int rc = settle(ctx, -1);
    if (rc) return rc;
    cudaSetDevice(ctx->device);
    cudaError_t e = ctx->waves.times(event_ms, traversal_ms);
    if (e != cudaSuccess) { cudaGetLastError(); return fail(ctx, Failure{SKG_ERR_CUDA, cudaGetErrorString(e)}); }
    if (waves) *waves = ctx->waves.waves();
    return SKG_OK;
}

int skg_reset_tallies(skg_ctx* ctx) {
    if (!ctx) return SKG_ERR_INVALID;
    int rc = settle(ctx, -1);
    if (rc) return rc;
    ctx->wave_count = 0;
    try {
        CK(cudaSetDevice(ctx->device));
        cudaStream_t s = ctx->stream;
        for (int i = 0; i < ctx->hs.ninstr; i++) {
            if (ctx->cube_len[i]) CK(cudaMemsetAsync(ctx->hs.instr[i].cube, 0, ctx->cube_len[i] * sizeof(double), s));
            CK(cudaMemsetAsync(ctx->hs.instr[i].sed, 0, ctx->sed_len[i] * sizeof(double), s));
        }
        size_t nlab = (size_t)ctx->ncells * ctx->nlambda;
        if (ctx->hs.labs_stel) CK(cudaMemsetAsync(ctx->hs.labs_stel, 0, nlab * sizeof(double), s));
        if (ctx->hs.labs_dust) CK(cudaMemsetAsync(ctx->hs.labs_dust, 0, nlab * sizeof(double), s));
        CK(cudaMemsetAsync(ctx->counters, 0, 10 * sizeof(unsigned long long), s));
        return SKG_OK;
    } catch (const Failure& f) { return fail(ctx, f); }
}

int skg_tally_sizes(const skg_ctx* ctx, int instr, int64_t* cube_len, int64_t* sed_len) {
    if (!ctx || instr < 0 || instr >= ctx->hs.ninstr) return SKG_ERR_INVALID;
    if (cube_len) *cube_len = ctx->cube_len[instr];
    if (sed_len) *sed_len = ctx->sed_len[instr];
    return SKG_OK;
}

int skg_read_instrument(skg_ctx* ctx, int instr, double* cube, double* sed) {
    if (!ctx || instr < 0 || instr >= ctx->hs.ninstr) return SKG_ERR_INVALID;
    int rc = skg_sync(ctx, -1);
    if (rc) return rc;
    try {
        if (cube && ctx->cube_len[instr])
            CK(cudaMemcpy(cube, ctx->hs.instr[instr].cube, ctx->cube_len[instr] * sizeof(double), cudaMemcpyDeviceToHost));
        if (sed) CK(cudaMemcpy(sed, ctx->hs.instr[instr].sed, ctx->sed_len[instr] * sizeof(double), cudaMemcpyDeviceToHost));
        return SKG_OK;
    } catch (const Failure& f) { return fail(ctx, f); }
}

int skg_read_instrument_device(skg_ctx* ctx, int instr, double* d_cube, double* d_sed, void* stream) {
    if (!ctx || instr < 0 || instr >= ctx->hs.ninstr) return SKG_ERR_INVALID;
    int rc = settle(ctx, -1);
    if (rc) return rc;
    try {
        CK(cudaSetDevice(ctx->device));
        cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
        if (d_cube && ctx->cube_len[instr])
            CK(cudaMemcpyAsync(d_cube, ctx->hs.instr[instr].cube, ctx->cube_len[instr] * sizeof(double),
                               cudaMemcpyDeviceToDevice, s));
        if (d_sed) CK(cudaMemcpyAsync(d_sed, ctx->hs.instr[instr].sed, ctx->sed_len[instr] * sizeof(double),
                                      cudaMemcpyDeviceToDevice, s));
        return SKG_OK;
    } catch (const Failure& f) { return fail(ctx, f); }
}

int skg_read_absorption(skg_ctx* ctx, double* labs_stellar, double* labs_dust) {
    if (!ctx) return SKG_ERR_INVALID;
    int rc = skg_sync(ctx, -1);
    if (rc) return rc;
    try {
        const size_t nc = (size_t)ctx->ncells, nl = (size_t)ctx->nlambda, n = nc * nl;
        // the device tables are wavelength-major ([ell][m]); the caller gets [m][ell]
        std::vector<double> t;
        auto read = [&](const double* dev, double* out) {
            if (!out) return;
            if (!dev) { std::memset(out, 0, n * sizeof(double)); return; }
            t.resize(n);
            CK(cudaMemcpy(t.data(), dev, n * sizeof(double), cudaMemcpyDeviceToHost));
            const size_t B = 64;                        // cache blocks of the transpose
            for (size_t m0 = 0; m0 < nc; m0 += B)
                for (size_t e0 = 0; e0 < nl; e0 += B)
                    for (size_t m = m0; m < std::min(nc, m0 + B); m++)
                        for (size_t e = e0; e < std::min(nl, e0 + B); e++) out[m * nl + e] = t[e * nc + m];
        };
        read(ctx->hs.labs_stel, labs_stellar);
        read(ctx->hs.labs_dust, labs_dust);
        return SKG_OK;
    } catch (const Failure& f) { return fail(ctx, f); }
}

int skg_read_counters(skg_ctx* ctx, skg_counters* out) {
    if (!ctx || !out) return SKG_ERR_INVALID;
    int rc = skg_sync(ctx, -1);
    if (rc && rc != SKG_ERR_STEP_BUDGET && rc != SKG_ERR_NAN_TAU) return rc;
    unsigned long long c[10];
    cudaMemcpy(c, ctx->counters, sizeof(c), cudaMemcpyDeviceToHost);
    out->packets = c[0]; out->steps = c[1]; out->traversals = c[2]; out->scatterings = c[3]; out->peeloffs = c[4];
    out->absorb_adds = c[5]; out->pixel_adds = c[6]; out->nbr_scanned = c[7]; out->fallbacks = c[8]; out->errors = c[9];
    out->waves = ctx->wave_count;
    return rc;
}

int skg_calc_dust_emission(skg_ctx* ctx, double* temperature) {
    if (!ctx) return SKG_ERR_INVALID;
    int rc = settle(ctx, -1);
    if (rc) return rc;
    try {
        CK(cudaSetDevice(ctx->device));
        REQUIRE(ctx->emit_cdf != nullptr, "dust emission is not enabled for this scene");
        cudaStream_t s = ctx->stream;
        CK(launch_dust_emission(ctx->grid, ctx->ds, ctx->Tv, ctx->planckabs, ctx->nT, ctx->labsbol, ctx->spectra,
                                ctx->temperature, s));
        CK(launch_emission_sources(ctx->ds, ctx->nlambda, (int)ctx->ncells, ctx->labsbol, ctx->spectra, ctx->emit_Lv,
                                   ctx->emit_cdf, ctx->emit_Ltot, ctx->scan_scratch, ctx->scan_bytes, s));
        if (temperature) CK(cudaMemcpyAsync(temperature, ctx->temperature, ctx->ncells * sizeof(double), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        return SKG_OK;
    } catch (const Failure& f) { return fail(ctx, f); }
}

int skg_absorbed_totals(skg_ctx* ctx, double* tot_stel, double* tot_dust) {
    if (!ctx) return SKG_ERR_INVALID;
    int rc = settle(ctx, -1);
    if (rc) return rc;
    try {
        CK(cudaSetDevice(ctx->device));
        cudaStream_t s = ctx->stream;
        size_t n = (size_t)ctx->ncells * ctx->nlambda;
        double h[2] = {0, 0};
        if (ctx->hs.labs_stel) CK(launch_sum(ctx->hs.labs_stel, n, ctx->sumbuf, s));
        if (ctx->hs.labs_stel) CK(cudaMemcpyAsync(&h[0], ctx->sumbuf, sizeof(double), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        if (ctx->hs.labs_dust) CK(launch_sum(ctx->hs.labs_dust, n, ctx->sumbuf + 1, s));
        if (ctx->hs.labs_dust) CK(cudaMemcpyAsync(&h[1], ctx->sumbuf + 1, sizeof(double), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        if (tot_stel) *tot_stel = h[0];
        if (tot_dust) *tot_dust = h[1];
        return SKG_OK;
    } catch (const Failure& f) { return fail(ctx, f); }
}

int skg_reset_dust_absorption(skg_ctx* ctx) {
    if (!ctx) return SKG_ERR_INVALID;
    int rc = settle(ctx, -1);
    if (rc) return rc;
    try {
        CK(cudaSetDevice(ctx->device));
        if (ctx->hs.labs_dust)
            CK(cudaMemsetAsync(ctx->hs.labs_dust, 0, (size_t)ctx->ncells * ctx->nlambda * sizeof(double), ctx->stream));
        return SKG_OK;
    } catch (const Failure& f) { return fail(ctx, f); }
}

// ---------------------------------------------------------------------------------------------
// trees

int skg_tree_build(const skg_scene* sc, int type, int min_level, int max_level, double max_mass_fraction,
                   int samples, uint64_t seed, int device, skg_tree** out) {
    *out = nullptr;
    skg_tree* T = new skg_tree();
    try {
        REQUIRE(sc && sc->ncomp > 0, "tree construction needs a dust distribution");
        REQUIRE(type == SKG_GRID_OCTREE || type == SKG_GRID_BINTREE, "tree type must be octree or k-d tree");
        REQUIRE(min_level >= 0 && max_level >= 2 && max_level > min_level && max_level <= 50, "invalid tree levels");
        REQUIRE(samples >= 10 && samples <= 1000, "sample count must be in [10,1000]");
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { cudaGetLastError(); throw Failure{SKG_ERR_NO_DEVICE, "no CUDA device"}; }
        CK(cudaSetDevice(device));
        cudaStream_t s;
        CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        Allocs A;
        std::vector<DevGeometry> dg(sc->ncomp);
        std::vector<double> norms(sc->ncomp);
        double total_mass = 0;
        for (int h = 0; h < sc->ncomp; h++) {
            dg[h] = make_geometry(A, sc->dust[h].geometry, s);
            norms[h] = sc->dust[h].norm; total_mass += norms[h];   // DustComp::mass() (DustComp.cpp:110-114)
        }
        DevGeometry* dgd = upload(A, dg.data(), dg.size(), s);
        double* nd = upload(A, norms.data(), norms.size(), s);
        Tree& t = T->t;
        t.type = type;
        t.ext[0] = sc->grid.xmin; t.ext[1] = sc->grid.ymin; t.ext[2] = sc->grid.zmin;
        t.ext[3] = sc->grid.xmax; t.ext[4] = sc->grid.ymax; t.ext[5] = sc->grid.zmax;
        Allocs B;
        size_t cap = 0;
        double *dbox = nullptr, *dm = nullptr, *dlo = nullptr, *dhi = nullptr;
        auto sample = [&](const std::vector<int>& ids, std::vector<double>& mass, std::vector<double>& rmin,
                          std::vector<double>& rmax) {
            size_t n = ids.size();
            if (n > cap) {
                B.release();
                cap = std::max(n, 2 * cap);
                dbox = B.alloc<double>(6 * cap); dm = B.alloc<double>(cap); dlo = B.alloc<double>(cap); dhi = B.alloc<double>(cap);
                if (!dbox || !dm || !dlo || !dhi) throw Failure{SKG_ERR_OOM, "device allocation failed"};
            }
            std::vector<double> hb(6 * n);
            for (size_t q = 0; q < n; q++) std::memcpy(&hb[6 * q], t.nodes[ids[q]].box, 6 * sizeof(double));
            CK(cudaMemcpyAsync(dbox, hb.data(), hb.size() * sizeof(double), cudaMemcpyHostToDevice, s));
            CK(launch_node_mass(dgd, nd, sc->ncomp, dbox, (int)n, samples, seed, (uint64_t)ids[0], dm, dlo, dhi, s));
            mass.resize(n); rmin.resize(n); rmax.resize(n);
            CK(cudaMemcpyAsync(mass.data(), dm, n * sizeof(double), cudaMemcpyDeviceToHost, s));
            CK(cudaMemcpyAsync(rmin.data(), dlo, n * sizeof(double), cudaMemcpyDeviceToHost, s));
            CK(cudaMemcpyAsync(rmax.data(), dhi, n * sizeof(double), cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
        };
        t.build(min_level, max_level, max_mass_fraction, 0.0, 0.0, total_mass, sample);
        CK(cudaStreamSynchronize(s));
        cudaStreamDestroy(s);
        t.finish(true);
        t.flatten();
        *out = T;
        return SKG_OK;
    } catch (const Failure& f) {
        delete T;
        return fail(nullptr, f);
    }
}

int skg_tree_from_splits(int type, double xmin, double ymin, double zmin, double xmax, double ymax, double zmax,
                         const uint8_t* split, int64_t nsplit, skg_tree** out) {
    *out = nullptr;
    if (type != SKG_GRID_OCTREE && type != SKG_GRID_BINTREE) { set_error("tree type must be octree or k-d tree"); return SKG_ERR_INVALID; }
    skg_tree* T = new skg_tree();
    Tree& t = T->t;
    t.type = type;
    t.ext[0] = xmin; t.ext[1] = ymin; t.ext[2] = zmin; t.ext[3] = xmax; t.ext[4] = ymax; t.ext[5] = zmax;
    t.build_from_splits(split, nsplit);
    t.finish(true);
    t.flatten();
    *out = T;
    return SKG_OK;
}

int skg_tree_sizes(const skg_tree* T, int32_t* nnodes, int32_t* ncells, int64_t* nnbr) {
    if (!T) return SKG_ERR_INVALID;
    if (nnodes) *nnodes = (int32_t)T->t.nodes.size();
    if (ncells) *ncells = T->t.ncells;
    if (nnbr) *nnbr = (int64_t)T->t.nbr.size();
    return SKG_OK;
}

int skg_tree_arrays(const skg_tree* T, double* node_box, int32_t* node_child, int32_t* node_father,
                    int32_t* node_cell, int8_t* node_dir, int64_t* nbr_offsets, int32_t* nbr_ids) {
    if (!T) return SKG_ERR_INVALID;
    const Tree& t = T->t;
    size_t n = t.nodes.size();
    if (node_box) std::memcpy(node_box, t.box.data(), 6 * n * sizeof(double));
    if (node_child) std::memcpy(node_child, t.child.data(), n * sizeof(int32_t));
    if (node_father) std::memcpy(node_father, t.father.data(), n * sizeof(int32_t));
    if (node_cell) std::memcpy(node_cell, t.cell.data(), n * sizeof(int32_t));
    if (node_dir) std::memcpy(node_dir, t.dir.data(), n * sizeof(int8_t));
    if (nbr_offsets) std::memcpy(nbr_offsets, t.nbroff.data(), t.nbroff.size() * sizeof(int64_t));
    if (nbr_ids) std::memcpy(nbr_ids, t.nbr.data(), t.nbr.size() * sizeof(int32_t));
    return SKG_OK;
}

int skg_tree_grid(const skg_tree* T, skg_grid* grid) {
    if (!T || !grid) return SKG_ERR_INVALID;
    T->t.fill_grid(grid);
    return SKG_OK;
}

int skg_tree_destroy(skg_tree* T) { delete T; return SKG_OK; }

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// batched launches

struct skg_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    Allocs A;
    Staging T;
    // pinned host mirrors of the tables (read by the copies of a replayed graph)
    BatchHeader* h_hdr = nullptr;
    WorkItem* h_items = nullptr;
    DevGrid* h_grids = nullptr;
    const DevScene** h_scenes = nullptr;
    int* h_ells = nullptr;
    cudaEvent_t copied = nullptr;          // the previous launch's tables have been read
    cudaGraphExec_t graph = nullptr;
    int g_type = -1, g_bk = -1, g_prec = -1, g_blocks = -1;
    size_t g_npool = 0;
    int g_waves = 0;                       // waves captured in the graph
    bool g_stale = false;                  // a replay needed more waves than captured
    cudaStream_t g_stream = nullptr;
    WaveRunner waves;
    uint64_t wave_count = 0;
    std::string error;
};

static int bfail(skg_batch* b, const Failure& f) {
    set_error(f.msg);
    if (b) b->error = f.msg;
    return f.code;
}

// Completes the batch's running phase (see settle for contexts).
static int bsettle(skg_batch* b, int timeout_ms) {
    if (!b->waves.pending()) return SKG_OK;
    cudaSetDevice(b->device);
    bool timed_out = false;
    cudaError_t e = b->waves.finish(timeout_ms, b->ev1, &timed_out);
    if (e != cudaSuccess) { cudaGetLastError(); return bfail(b, Failure{SKG_ERR_CUDA, cudaGetErrorString(e)}); }
    if (timed_out) return bfail(b, Failure{SKG_ERR_TIMEOUT, "timed out waiting for the device"});
    b->wave_count = b->waves.waves();
    if (b->graph && b->waves.waves() > b->g_waves) b->g_stale = true;
    return SKG_OK;
}

extern "C" {

int skg_batch_create(int device, int max_slots, int max_items, int max_ells, skg_batch** out) {
    *out = nullptr;
    skg_batch* b = new skg_batch();
    try {
        REQUIRE(max_slots >= 1 && max_slots <= MAX_SLOTS, "1..64 slots per batch");
        REQUIRE(max_items >= 1 && max_ells >= 1, "batch table sizes must be positive");
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { cudaGetLastError(); throw Failure{SKG_ERR_NO_DEVICE, "no CUDA device"}; }
        REQUIRE(device >= 0 && device < ndev, "device index out of range");
        b->device = device;
        CK(cudaSetDevice(device));
        CK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
        CK(cudaEventCreate(&b->ev0)); CK(cudaEventCreate(&b->ev1));
        CK(cudaEventCreateWithFlags(&b->copied, cudaEventDisableTiming));
        b->T.alloc(b->A, max_items, max_slots, max_ells);
        CK(cudaMemset(b->T.counters, 0, 10 * sizeof(unsigned long long)));
        CK(cudaMemset(b->T.err, 0, sizeof(unsigned)));
        CK(cudaMallocHost((void**)&b->h_hdr, sizeof(BatchHeader)));
        CK(cudaMallocHost((void**)&b->h_items, max_items * sizeof(WorkItem)));
        CK(cudaMallocHost((void**)&b->h_grids, max_slots * sizeof(DevGrid)));
        CK(cudaMallocHost((void**)&b->h_scenes, max_slots * sizeof(void*)));
        CK(cudaMallocHost((void**)&b->h_ells, max_ells * sizeof(int)));
        CK(cudaEventRecord(b->copied, b->stream));
        *out = b;
        return SKG_OK;
    } catch (const Failure& f) {
        int rc = bfail(nullptr, f);
        skg_batch_destroy(b);
        return rc;
    }
}

int skg_batch_destroy(skg_batch* b) {
    if (!b) return SKG_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->g_stream) cudaStreamSynchronize(b->g_stream);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    if (b->g_stream) cudaStreamDestroy(b->g_stream);
    b->A.release();
    if (b->h_hdr) cudaFreeHost(b->h_hdr);
    if (b->h_items) cudaFreeHost(b->h_items);
    if (b->h_grids) cudaFreeHost(b->h_grids);
    if (b->h_scenes) cudaFreeHost((void*)b->h_scenes);
    if (b->h_ells) cudaFreeHost(b->h_ells);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->copied) cudaEventDestroy(b->copied);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return SKG_OK;
}

int skg_batch_run(skg_batch* b, int phase, const skg_work* work, int nwork, const skg_run_opts* opts, int flags,
                  void* stream) {
    if (!b) return SKG_ERR_INVALID;
    int rc = bsettle(b, -1);
    if (rc) return rc;
    try {
        CK(cudaSetDevice(b->device));
        REQUIRE(phase >= SKG_PHASE_STELLAR && phase <= SKG_PHASE_DUST_EMISSION, "unknown phase");
        REQUIRE(nwork >= 0, "negative work item count");
        if (nwork > b->T.max_items) throw Failure{SKG_ERR_CAPACITY, "more work items than the batch was created for"};
        cudaStream_t s = stream ? (cudaStream_t)stream : b->stream;
        // the pinned tables may still be read by the previous launch's copies
        CK(cudaEventSynchronize(b->copied));
        int nslots = 0, nells = 0, gtype = -1, gbk = -1;
        uint64_t total = 0;
        std::vector<skg_ctx*> slots;
        for (int i = 0; i < nwork; i++) {
            const skg_work& w = work[i];
            REQUIRE(w.ctx != nullptr && w.ells && w.nell > 0, "work item needs a context and wavelengths");
            REQUIRE(w.ctx->device == b->device, "all contexts must live on the batch's device");
            REQUIRE(w.count <= w.npp, "packet range exceeds the packet count");
            if (gtype < 0) gtype = w.ctx->grid.type;
            auto tree = [](int t) { return t == SKG_GRID_OCTREE || t == SKG_GRID_BINTREE; };
            REQUIRE(w.ctx->grid.type == gtype || (tree(gtype) && tree(w.ctx->grid.type)),
                    "a batch holds one kind of grid");
            const int bk = tree_walk_of(w.ctx->grid);
            if (gbk < 0) gbk = bk;
            if (gtype == SKG_GRID_CARTESIAN) gbk = std::min(gbk, bk);   // the plane tables serve every grid
            else if (tree(gtype)) REQUIRE(bk == gbk, "a batch holds trees of one walk kind (Bookkeeping search, rope or lattice records)");
            if (phase != SKG_PHASE_STELLAR) REQUIRE(w.ctx->emit_cdf != nullptr, "dust phases need dust emission enabled");
            int slot = -1;
            for (int q = 0; q < nslots; q++) if (slots[q] == w.ctx) slot = q;
            if (slot < 0) {
                if (!(nslots < b->T.max_slots)) throw Failure{SKG_ERR_CAPACITY, "too many distinct simulations for this batch"};
                slot = nslots++;
                slots.push_back(w.ctx);
                DevGrid g = w.ctx->grid;
                if (opts && opts->max_steps > 0) g.max_steps = opts->max_steps;
                b->h_grids[slot] = g;
                b->h_scenes[slot] = w.ctx->ds;
            }
            if (!(nells + w.nell <= b->T.max_ells)) throw Failure{SKG_ERR_CAPACITY, "too many wavelength entries for this batch"};
            WorkItem& W = b->h_items[i];
            std::memset(&W, 0, sizeof(W));
            W.slot = slot; W.nell = w.nell; W.ell0 = nells; W.npp_total = w.npp; W.first = w.first; W.count = w.count;
            W.seed = w.seed; W.begin = total;
            for (int e = 0; e < w.nell; e++) {
                REQUIRE(w.ells[e] >= 0 && w.ells[e] < w.ctx->nlambda, "wavelength index out of range");
                b->h_ells[nells + e] = w.ells[e];
            }
            nells += w.nell;
            total += (uint64_t)w.nell * w.count;
        }
        *b->h_hdr = BatchHeader{phase, nslots, nwork, 0, total};
        int precision = opts ? opts->precision : SKG_PREC_FP32;
        int blocks = opts ? opts->blocks : 0;
        REQUIRE(!opts || opts->pool >= 0, "negative packet pool");
        REQUIRE(!opts || opts->precision == SKG_PREC_FP32 || opts->precision == SKG_PREC_FP64, "unknown precision");
        // the pool: enough records for the batch up to the pool limit, rounded up to a power of two
        // so that replays of a captured graph keep fitting
        const size_t pool_max = (opts && opts->pool > 0) ? (size_t)opts->pool : ((size_t)1 << 21);
        size_t npool = 1;
        while (npool < total && npool < pool_max) npool <<= 1;
        npool = std::min(npool, pool_max);
        int ngroups = 0;
        for (skg_ctx* c : slots) ngroups = std::max(ngroups, c->hs.ngroups);
        if (total == 0) return SKG_OK;
        CK(b->waves.reserve(npool, ngroups, gtype));
        REQUIRE(!opts || (opts->refill >= 0 && opts->refill <= 32), "refill lanes must be in 0..32");
        RunParams P = b->T.params((opts && opts->max_scatt > 0) ? opts->max_scatt : 100000, opts ? opts->refill : 0);
        Staging& T = b->T;
        auto enqueue = [&](cudaStream_t q) {
            CK(cudaMemcpyAsync(T.hdr, b->h_hdr, sizeof(BatchHeader), cudaMemcpyHostToDevice, q));
            CK(cudaMemcpyAsync(T.items, b->h_items, T.max_items * sizeof(WorkItem), cudaMemcpyHostToDevice, q));
            CK(cudaMemcpyAsync(T.grids, b->h_grids, T.max_slots * sizeof(DevGrid), cudaMemcpyHostToDevice, q));
            CK(cudaMemcpyAsync(T.scenes, b->h_scenes, T.max_slots * sizeof(void*), cudaMemcpyHostToDevice, q));
            CK(cudaMemcpyAsync(T.ells, b->h_ells, T.max_ells * sizeof(int), cudaMemcpyHostToDevice, q));
            CK(cudaMemsetAsync(T.work, 0, sizeof(unsigned long long), q));
            CK(cudaMemsetAsync(T.err, 0, sizeof(unsigned), q));
            // every slot's DevGrid is copied into shared memory: size for the batch's capacity
            CK(b->waves.begin(P, gtype < 0 ? SKG_GRID_CARTESIAN : gtype, gbk < 0 ? TW_ROPE : gbk, precision, T.max_slots, npool,
                              blocks, q));
        };
        CK(cudaEventRecord(b->ev0, s));
        if (flags & SKG_BATCH_GRAPH) {
            bool same = b->graph && !b->g_stale && b->g_type == gtype && b->g_bk == gbk && b->g_prec == precision &&
                        b->g_blocks == blocks && b->g_npool == npool;
            if (!same) {
                if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
                if (!b->g_stream) CK(cudaStreamCreateWithFlags(&b->g_stream, cudaStreamNonBlocking));
                cudaGraph_t gr;
                CK(cudaStreamBeginCapture(b->g_stream, cudaStreamCaptureModeThreadLocal));
                enqueue(b->g_stream);
                CK(cudaStreamEndCapture(b->g_stream, &gr));
                cudaError_t e = cudaGraphInstantiate(&b->graph, gr, 0);
                cudaGraphDestroy(gr);
                CK(e);
                b->g_type = gtype; b->g_bk = gbk; b->g_prec = precision; b->g_blocks = blocks; b->g_npool = npool;
                b->g_waves = b->waves.waves(); b->g_stale = false;
            }
            CK(cudaGraphLaunch(b->graph, s));
            b->waves.replayed(s, b->g_waves);       // the replay runs the captured waves on s
        } else {
            enqueue(s);
        }
        CK(cudaEventRecord(b->ev1, s));
        CK(cudaEventRecord(b->copied, s));
        return SKG_OK;
    } catch (const Failure& f) { return bfail(b, f); }
}

int skg_batch_sync(skg_batch* b, int timeout_ms) {
    if (!b) return SKG_ERR_INVALID;
    int rc = bsettle(b, timeout_ms);
    if (rc) return rc;
    cudaSetDevice(b->device);
    auto t0 = std::chrono::steady_clock::now();
    while (true) {
        cudaError_t e = cudaEventQuery(b->ev1);
        if (e == cudaSuccess) break;
        if (e != cudaErrorNotReady) { cudaGetLastError(); return bfail(b, Failure{SKG_ERR_CUDA, cudaGetErrorString(e)}); }
        if (timeout_ms >= 0 && std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count() > timeout_ms)
            return bfail(b, Failure{SKG_ERR_TIMEOUT, "timed out waiting for the device"});
        std::this_thread::sleep_for(std::chrono::microseconds(100));
    }
    unsigned err = 0;
    cudaMemcpy(&err, b->T.err, sizeof(unsigned), cudaMemcpyDeviceToHost);
    if (err & ERR_NAN_TAU) return bfail(b, Failure{SKG_ERR_NAN_TAU, "The optical depth along the path is not a positive number"});
    if (err & (ERR_STEP_BUDGET | ERR_SCATT_BUDGET)) return bfail(b, Failure{SKG_ERR_STEP_BUDGET, "a packet exceeded its step or scattering budget"});
    return SKG_OK;
}

int skg_batch_counters(skg_batch* b, skg_counters* out) {
    if (!b || !out) return SKG_ERR_INVALID;
    int rc = skg_batch_sync(b, -1);
    unsigned long long c[10];
    cudaMemcpy(c, b->T.counters, sizeof(c), cudaMemcpyDeviceToHost);
    out->packets = c[0]; out->steps = c[1]; out->traversals = c[2]; out->scatterings = c[3]; out->peeloffs = c[4];
    out->absorb_adds = c[5]; out->pixel_adds = c[6]; out->nbr_scanned = c[7]; out->fallbacks = c[8]; out->errors = c[9];
    out->waves = b->wave_count;
    return rc;
}

int skg_batch_last_ms(skg_batch* b, float* ms) {
    if (!b || !ms) return SKG_ERR_INVALID;
    int rc = bsettle(b, -1);
    if (rc) return rc;
    cudaSetDevice(b->device);
    cudaError_t e = cudaEventSynchronize(b->ev1);
    if (e != cudaSuccess) { cudaGetLastError(); return bfail(b, Failure{SKG_ERR_CUDA, cudaGetErrorString(e)}); }
    cudaEventElapsedTime(ms, b->ev0, b->ev1);
    return SKG_OK;
}


/* ---- path harness without device allocation ------------------------------------------------
   skg_trace_paths allocates its staging and scan buffers on every call.  Callers that own all
   of the device memory themselves -- a serving loop that reserves a fixed share of HBM up front,
   or a host framework whose allocator must stay the only one, where a cudaMalloc in the middle
   of a request would synchronise the device and could fail on a fragmented heap -- cannot use
   it.  skg_trace_paths_noalloc takes device buffers from the caller and keeps its only scratch
   (the per-ray segment counts, turned in place into offsets, and the scan's block totals) in the
   file-scope array below, so the call performs no allocation at all.  The same count and write
   kernels as skg_trace_paths produce the segments, hence the results are identical. */
}  // extern "C"

namespace {

constexpr int NA_SCAN = 1024;                                         // rays per scan block
constexpr int64_t NA_MAX_RAYS = SKG_NOALLOC_MAX_RAYS;
constexpr int64_t NA_MAX_BLOCKS = NA_MAX_RAYS / NA_SCAN;
static_assert(NA_MAX_RAYS % NA_SCAN == 0 && NA_MAX_BLOCKS <= NA_SCAN, "one block scans the block totals");

// [0, NA_MAX_RAYS]: segment count of ray i, later the write offset of ray i (clamped to the
// caller's capacity); [NA_MAX_RAYS + 1, +NA_MAX_BLOCKS): scan totals per block.  Every entry a
// call reads is written earlier in that call, so nothing here has to start at zero.
// 8 MiB + 8 KiB per device.
static __device__ __align__(256) int64_t g_noalloc_scratch[NA_MAX_RAYS + 1 + NA_MAX_BLOCKS];

std::mutex g_noalloc_mutex;
int64_t* g_noalloc_addr[64] = {};

__device__ int64_t na_block_inclusive_scan(int64_t v) {
    __shared__ int64_t warp_tot[NA_SCAN / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int o = 1; o < 32; o <<= 1) {
        int64_t u = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += u;
    }
    if (lane == 31) warp_tot[w] = v;
    __syncthreads();
    if (w == 0) {
        int64_t t = lane < (int)(blockDim.x >> 5) ? warp_tot[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            int64_t u = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += u;
        }
        warp_tot[lane] = t;
    }
    __syncthreads();
    return v + (w > 0 ? warp_tot[w - 1] : 0);
}

// inclusive scan of the counts inside each block -> offsets[i + 1]; block totals -> scratch
__global__ void na_scan_blocks(const int64_t* __restrict__ counts, int64_t n, int64_t* offsets, int64_t* block_tot) {
    int64_t i = (int64_t)blockIdx.x * NA_SCAN + threadIdx.x;
    int64_t v = na_block_inclusive_scan(i < n ? counts[i] : 0);
    if (i < n) offsets[i + 1] = v;
    if (threadIdx.x == NA_SCAN - 1) block_tot[blockIdx.x] = v;
}

// exclusive scan of the block totals (one block); flags a total above the capacity
__global__ void na_scan_totals(int64_t* block_tot, int nblocks, int64_t capacity, unsigned* err) {
    int64_t t = threadIdx.x < nblocks ? block_tot[threadIdx.x] : 0;
    int64_t inc = na_block_inclusive_scan(t);
    if (threadIdx.x < nblocks) block_tot[threadIdx.x] = inc - t;
    if (threadIdx.x == nblocks - 1 && inc > capacity) atomicOr(err, ERR_CAPACITY);
}

// final offsets for the caller, and the same offsets clamped to the capacity for the write pass
// (a ray whose segments do not fit then stops at the clamp and flags the overflow)
__global__ void na_add_offsets(int64_t* offsets, const int64_t* __restrict__ block_pre, int64_t n,
                               int64_t capacity, int64_t* woff) {
    int64_t i = (int64_t)blockIdx.x * NA_SCAN + threadIdx.x;
    if (i == 0) { offsets[0] = 0; woff[0] = 0; }
    if (i >= n) return;
    int64_t o = offsets[i + 1] + block_pre[blockIdx.x];
    offsets[i + 1] = o;
    woff[i + 1] = o < capacity ? o : capacity;
}

}  // namespace

extern "C" {

int skg_trace_paths_noalloc(skg_ctx* ctx, const double* d_r, const double* d_k, int64_t n, int precision,
                            int32_t* d_cells, double* d_ds, int64_t* d_offsets, int64_t capacity, void* stream) {
    if (n > NA_MAX_RAYS)
        return fail(ctx, Failure{SKG_ERR_CAPACITY, "skg_trace_paths_noalloc: " + std::to_string(n) +
                                 " rays exceed the per-call maximum of " + std::to_string(NA_MAX_RAYS)});
    if (!ctx || n < 0 || capacity < 0 || !d_offsets || (n > 0 && (!d_r || !d_k)) || (capacity > 0 && (!d_cells || !d_ds)))
        return fail(ctx, Failure{SKG_ERR_INVALID, "skg_trace_paths_noalloc: invalid arguments"});
    if (precision != SKG_PREC_FP32 && precision != SKG_PREC_FP64)
        return fail(ctx, Failure{SKG_ERR_INVALID, "skg_trace_paths_noalloc: unknown precision"});
    // a phase still running on the context finishes first (its waves complete; its error flags
    // stay in the phase word for skg_sync)
    int rc = settle(ctx, -1);
    if (rc) return rc;
    try {
        CK(cudaSetDevice(ctx->device));
        REQUIRE(ctx->device >= 0 && ctx->device < 64, "device ordinal out of range");
        int64_t* scratch;
        {
            // the scratch address of this device, looked up once (with the device current)
            std::lock_guard<std::mutex> lock(g_noalloc_mutex);
            if (!g_noalloc_addr[ctx->device]) {
                void* p = nullptr;
                CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
                g_noalloc_addr[ctx->device] = (int64_t*)p;
            }
            scratch = g_noalloc_addr[ctx->device];
        }
        int64_t* block_tot = scratch + NA_MAX_RAYS + 1;
        cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
        CK(cudaMemsetAsync(ctx->herr, 0, sizeof(unsigned), s));
        if (n == 0) {
            CK(cudaMemsetAsync(d_offsets, 0, sizeof(int64_t), s));
        } else {
            int nblocks = (int)((n + NA_SCAN - 1) / NA_SCAN);
            CK(launch_count_segments(ctx->grid, d_r, d_k, n, precision, scratch, ctx->herr, s));
            na_scan_blocks<<<nblocks, NA_SCAN, 0, s>>>(scratch, n, d_offsets, block_tot);
            CK(cudaGetLastError());
            na_scan_totals<<<1, NA_SCAN, 0, s>>>(block_tot, nblocks, capacity, ctx->herr);
            CK(cudaGetLastError());
            na_add_offsets<<<nblocks, NA_SCAN, 0, s>>>(d_offsets, block_tot, n, capacity, scratch);
            CK(cudaGetLastError());
            CK(launch_write_segments(ctx->grid, d_r, d_k, n, precision, scratch, d_cells, d_ds, ctx->herr, s));
        }
        // skg_sync waits for this point of the caller's stream before it reads the harness flags
        CK(cudaEventRecord(ctx->hev, s));
        ctx->hev_pending = true;
        return SKG_OK;
    } catch (const Failure& f) { return fail(ctx, f); }
}

}  // extern "C"
