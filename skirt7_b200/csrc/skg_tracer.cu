// skg_tracer.cu -- the wavefront photon-packet tracer.
//
// One phase (stellar emission, dust self-absorption or dust emission) of a batch of wavelengths of
// one or more simulations replaces Parallel::call(this, &dostellaremissionchunk, Nlambda, Nchunks)
// (MonteCarloSimulation.cpp:241-295) and the two dust chunk bodies
// (PanMonteCarloSimulation.cpp:191-346).  The life cycle of a packet,
//
//   launch -> peel-off (emission) -> path: absorption, escape fraction, termination test, forced
//   interaction point -> propagate -> peel-off (scattering) -> scatter -> path -> ...
//
// is cut at its traversals.  The packets in flight sit in a pool of 128-byte records.  Each wave
// runs these kernels:
//   event_kernel  one thread per record: detects the peel-offs walked in the previous wave and
//                 lists the packets at their interaction point and the free records;
//   launch_kernel one thread per listed record: moves a packet to its interaction point, writes
//                 its scattering peel-offs and scatters it, or launches a new packet into a free
//                 record; then appends the packet's next traversals to the wave's job list (one
//                 peel-off job per direction group and one path job);
//   trav_kernel   persistent, launched twice (the path jobs, then the peel-off jobs in a lean
//                 instantiation); each lane takes jobs one after another and walks them:
//                 peel-off  accumulates the optical depth towards an observer
//                           (DustSystem::opticaldepth, DustSystem.cpp:960-976);
//                 path      streams kappa*rho*ds into the FP64 cumulative optical depth and the
//                           per-cell absorption tallies (simulateescapeandabsorption, :432-509),
//                           applies the escape fraction and the termination test, samples the
//                           interaction optical depth (simulatepropagation, :513-531) and re-walks
//                           the path to the segment where the cumulative optical depth passes it,
//                           interpolating inside it (DustGridPath::pathlength, DustGridPath.cpp:162-173).
// The traversal kernel holds nothing but the walk, so it keeps few registers, no local memory and
// a small instruction footprint; the divergent event code runs once per packet per wave in a
// kernel of its own.  Instruments seen from the same direction share one peel-off traversal
// (identical optical depth; the reference recomputes it per instrument).
#include "skg_scene.cuh"
#include "skg_internal.h"
#include "skg_wave.h"
#include <cstring>
#include <type_traits>

#include <chrono>
#include <cstdlib>
#include <thread>

namespace skg {

#ifndef SKG_TRAV_MIN_BLOCKS
#define SKG_TRAV_MIN_BLOCKS 4
#endif
// The traversal pass as two kernels: the path jobs, then the peel-off jobs in an instantiation
// that holds the optical depth alone (no spills at 64 registers).  Octree disk, 10^7 packets:
// 202.5 ms against 214.2 ms for one kernel over both (Voronoi disk: 1357 against 1421 ms); the
// peel-off kernel at 5 or 6 blocks per SM (48 or 40 registers, spilling) is slower (219, 240 ms).
#ifndef SKG_PATH_MIN_BLOCKS
#define SKG_PATH_MIN_BLOCKS 4
#endif
#ifndef SKG_VOR_PATH_MIN_BLOCKS
#define SKG_VOR_PATH_MIN_BLOCKS 3
#endif
#ifndef SKG_PEEL_MIN_BLOCKS
#define SKG_PEEL_MIN_BLOCKS 4
#endif
#ifndef SKG_SPLIT_TRAV
#define SKG_SPLIT_TRAV 1
#endif
// programmatic dependent launch of the peel-off-job kernel after the path-job kernel
#ifndef SKG_PDL
#define SKG_PDL 1
#endif
// the event pass at 4 blocks of 256 per SM (64 registers, spilling part of the packet record):
// its divergent, latency-bound code gains more from the warps than it loses to the spills
// (octree disk, 10^7 packets: 34.6 ms against 45.2 ms at 2 blocks and 126 registers)
// packets at their interaction point and free records are scattered and relaunched by a pass of
// their own after the event pass, every lane of its warps doing the same work (octree disk, 10^7
// packets: phase 177.7 against 194.4 ms in one event pass; Cartesian 87.0 against 90.7 ms)
#ifndef SKG_LAUNCH_KERNEL
#define SKG_LAUNCH_KERNEL 1
#endif
#ifndef SKG_EVENT_MIN_BLOCKS
#define SKG_EVENT_MIN_BLOCKS 4
#endif
// threads per event-pass block: a block's slot on an SM is held until its slowest record is done,
// so small blocks free slots sooner (octree disk, 10^7 packets: event pass 29.5 ms with 64 threads,
// 32.4 with 128, 34.6 with 256)
#ifndef SKG_EVENT_THREADS
#define SKG_EVENT_THREADS 64
#endif
// a lane whose job ended takes the next one when this many lanes of its warp (or all of its live
// lanes) wait for one: the job start (job, packet record, start leaf: dependent loads) is then paid
// once for several lanes instead of stalling the warp for each (8 measured fastest of 1-32 on the
// octree disk: traversal pass 275 ms against 336 ms at 1 per 10^7 packets)
#ifndef SKG_REFILL_LANES
#define SKG_REFILL_LANES 8
#endif
// lanes whose path walk ended run the end of the path (escape fraction, termination test, the
// interaction sampling: long, divergent FP64 code) once this many lanes of the warp wait for it,
// or no lane is walking.  Per 10^7 packets, traversal pass at 1 / 4 / 8 / 16: octree disk 193 /
// 176 / 170 / 174 ms; at 1 / 8: Cartesian 95 / 71 ms, k-d tree 224 / 201 ms, Voronoi 1212 / 1186 ms.
#ifndef SKG_AFTER_LANES
#define SKG_AFTER_LANES 8
#endif
#ifndef SKG_REFILL_PEEL
#define SKG_REFILL_PEEL SKG_REFILL_LANES
#endif
// checkpoints of a path's walk (FP32 steppers that can resume): every SKG_CKPT_STRIDE cell steps,
// up to SKG_CKPT_N per packet record, the walk stores its state with the optical depth and path
// length so far; the re-walk to the interaction point then starts at the last checkpoint below the
// interaction optical depth (at most one stride of cell steps) instead of at the path's start
#ifndef SKG_CKPT
#define SKG_CKPT 1
#endif
// the scatter-and-launch pass's grid: the blocks resident at once (1), or 16 per SM (0);
// event + launch passes of a 10^7-packet octree-disk phase 13.3 against 14.4 ms
#ifndef SKG_LAUNCH_OCC
#define SKG_LAUNCH_OCC 1
#endif
// the event pass's grid for pools of at most this many records of a Cartesian grid: the blocks resident at once,
// striding over the pool (the per-block counter and SED flushes then happen once per resident
// block); larger pools: one thread per record.  Event pass of a 10^7-packet phase, pool 2^21:
// Cartesian disk 15.7 against 16.8 ms, a batch of 24 fit variants 560.7 against 566.6 ms (whole
// batch); pool 2^23 (2·10^6 packets per wavelength): octree disk 156 against 139 ms, k-d tree disk
// 190 against 188 ms -- so the stride only up to 2^21
#ifndef SKG_EVENT_STRIDE_POOL
#define SKG_EVENT_STRIDE_POOL (1 << 21)
#endif
// cell steps a lane takes per pass of the traversal loop (the warp's refill and end-of-path votes
// run once per pass): peel-off-job kernel, path-job kernel.  Traversal pass of a 10^7-packet
// phase (octree disk / Cartesian disk): 1 and 1: 161 / 69.1 ms; 2 and 1: 156 / 68.6; 2 and 2: 153 /
// 68.1; 2 and 3: 152.4 / 67.0; 2 and 4: 151.3 / 66.4; 3 or 4 steps in the peel-off kernel spilled
// then: 165 / 68.3.  With the per-axis rope the peel-off kernel no longer spills at 3 or 4, and at
// 2·10^6 packets per wavelength 3 and 4 take the octree disk 1360 ms against 1367 at 2 and 4 (4 and
// 4: 1365, 2 and 6: 1404); 3 and 4 against 2 and 4 elsewhere: Cartesian disk 61.2 / 61.7, k-d tree
// disk 1730 / 1734, Voronoi disk 252.8 / 253.4 ms, a batch of 24 fit variants 566 / 571 ms
#ifndef SKG_INNER_STEPS
#define SKG_INNER_STEPS 3
#endif
#ifndef SKG_INNER_PATH
#define SKG_INNER_PATH 4
#endif
#ifndef SKG_CKPT_N
#define SKG_CKPT_N 32
#endif
#ifndef SKG_CKPT_STRIDE
#define SKG_CKPT_STRIDE 16
#endif

enum Cnt : int { C_PACKETS = 0, C_STEPS, C_TRAV, C_SCATT, C_PEEL, C_ABS, C_PIX, C_NBR, C_FB, C_ERR, C_N };

template<typename R> SKG_D double rho_load(const DevScene& S, size_t i);
template<> SKG_D double rho_load<double>(const DevScene& S, size_t i) { return __ldg(S.rho + i); }
template<> SKG_D double rho_load<float>(const DevScene& S, size_t i) { return (double)__ldg(S.rhof + i); }

// KappaRho call-back (DustSystem.cpp:459-485)
template<typename R> SKG_D double kappa_rho(const DevScene& S, int m, int ell) {
    if (m < 0) return 0.0;
    if (S.ncomp == 1) return S.kext[ell] * rho_load<R>(S, (size_t)m);
    double r = 0;
    for (int h = 0; h < S.ncomp; h++) r += S.kext[h * S.nlambda + ell] * rho_load<R>(S, (size_t)h * S.ncells + m);
    return r;
}

// Does the stepper carry the density of the step's cell in its leaf record (a data member rho),
// or not (a static constant rho = -1)?
template<typename St> struct EmbeddedRho {
    static constexpr bool value = !std::is_same<decltype(&St::rho), const float*>::value;
};

// kappa*rho of a cell step.  One dust component: kappa_ext of the job's wavelength is held by the
// job (kext1 >= 0) and multiplied in FP32 with the density embedded in the leaf record (tree
// walks), or, in the FP32 walks without records (Cartesian, Voronoi), with the FP32 density table,
// instead of reading the scene's tables every step; the FP64 walks keep the FP64 product of
// KappaRho.  Resolved at compile time per stepper: a run-time choice between the two made the
// lattice walk load the table every step as well (octree traversal pass 7819 against 7212 ms).
template<typename R, typename St>
SKG_D double step_kr(const DevScene& S, const St& st, float kext1, int m, int ell) {
    if constexpr (sizeof(R) == 4 && !EmbeddedRho<St>::value) {
        if (kext1 >= 0.f) return (double)(kext1 * __ldg(S.rhof + m));
        return kappa_rho<R>(S, m, ell);
    } else {
        return (kext1 >= 0.f && st.rho >= 0.f) ? (double)(kext1 * st.rho) : kappa_rho<R>(S, m, ell);
    }
}

// Optical depth of a cell step.  SKG_DTAU32: one dust component on an FP32 walk forms the step's
// kappa*rho*ds in FP32 (the geometry's precision) before the FP64 sum (traversal pass of a phase,
// octree disk 1387 against 1385 ms, k-d tree disk 1745 against 1744 ms: off).
#ifndef SKG_DTAU32
#define SKG_DTAU32 0
#endif
template<typename R, typename St>
SKG_D double step_dtau(const DevScene& S, const St& st, float kext1, int m, int ell, R ds) {
#if SKG_DTAU32
    if constexpr (sizeof(R) == 4) {
        if (kext1 >= 0.f) {
            float r;
            if constexpr (EmbeddedRho<St>::value) r = st.rho; else r = __ldg(S.rhof + m);
            return (double)(kext1 * r * ds);
        }
    }
#endif
    return step_kr<R>(S, st, kext1, m, ell) * (double)ds;
}

// Instrument::detect for the members of one direction group after the shared traversal
// (SEDInstrument.cpp:32-42, FrameInstrument.cpp:33-47, SimpleInstrument.cpp:35-49,
// FullInstrument.cpp:109-177).  SED bins go to the block's private copy `psed` when it is given
// (every packet of a wavelength adds to the same SED bin: global atomics would serialise on it).
// Returns the number of tally updates.
// detect_group inlined into the event kernel: its call kept a 240-byte stack frame there (972
// bytes of spill loads per thread at 64 registers against 52 inlined); event pass of a
// 10^7-packet phase 14.3 against 16.1 ms (octree disk)
#ifndef SKG_DETECT_INLINE
#define SKG_DETECT_INLINE 1
#endif
// frame pixel tallies: lanes of a warp that add to the same pixel sum their values over the warp
// first and one of them adds (1), or every lane adds its own value (0).  Octree disk, 5*10^8
// packets: phase 7870 ms with the aggregation against 7850-7930 ms without, event pass 652 against
// 632-640 ms -- lanes of a warp rarely hit one pixel (their packets sit anywhere in the galaxy),
// so the match costs more than the atomics it saves; off by default.
#ifndef SKG_WARP_AGG
#define SKG_WARP_AGG 0
#endif
SKG_D void frame_add(double* addr, double v) {
#if SKG_WARP_AGG
    const unsigned act = __activemask();
    const unsigned peers = __match_any_sync(act, (unsigned long long)addr);
    if (peers & (peers - 1)) {
        double s = 0;
        for (unsigned m = peers; m; m &= m - 1) s += __shfl_sync(peers, v, __ffs(m) - 1);
        v = s;
    }
    if ((int)(threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(addr, v);
#else
    atomicAdd(addr, v);
#endif
}

#if SKG_DETECT_INLINE
__device__ __forceinline__
#else
__device__ __noinline__
#endif
int detect_group(const DevScene& S, int grp, int ell, double Lpeel, double tau,
                                         int nscatt_peel, bool stellar, int comp, double x, double y, double z,
                                         double* psed) {
    double Lextf = Lpeel * exp(-tau);
    const int nl = S.nlambda;
    int adds = 0;
    for (int q = S.group_start[grp]; q < S.group_start[grp + 1]; q++) {
        const int iq = S.group_instr[q];
        const DevInstr& I = S.instr[iq];
        auto sed_add = [&](int c, double v) {
            if (psed) atomicAdd(psed + S.sed_base[iq] + c * nl + ell, v);
            else atomicAdd(I.sed + (size_t)c * nl + ell, v);
            adds++;
        };
        int l = (I.type == SKG_INSTR_SED) ? -1 : pixel_on_detector(I, x, y, z);
        size_t fp = (size_t)I.nxp * I.nyp;
        if (I.type == SKG_INSTR_FRAME) {
            if (l >= 0) {
                frame_add(I.cube + (size_t)ell * fp + l, Lextf); adds++;
                // the frame of the packet's stellar component (component 1 + comp)
                if (I.ncomp > 1 && comp >= 0) { frame_add(I.cube + ((size_t)(1 + comp) * nl + ell) * fp + l, Lextf); adds++; }
            }
        } else if (I.type == SKG_INSTR_SED) {
            sed_add(0, Lextf);
        } else if (I.type == SKG_INSTR_SIMPLE) {
            sed_add(0, Lextf);
            if (l >= 0) { atomicAdd(I.cube + (size_t)ell * fp + l, Lextf); adds++; }
        } else {
            auto add = [&](int c, double v) {
                sed_add(c, v);
                if (l >= 0) { atomicAdd(I.cube + ((size_t)c * nl + ell) * fp + l, v); adds++; }
            };
            add(SKG_FULL_TOT, Lextf);
            if (stellar) {
                if (nscatt_peel == 0) { add(SKG_FULL_TRA, Lpeel); if (S.ncomp) add(SKG_FULL_STRDIR, Lextf); }
                else {
                    add(SKG_FULL_STRSCA, Lextf);
                    if (nscatt_peel <= I.nscatt_levels) add(SKG_FULL_NBASE + nscatt_peel - 1, Lextf);
                }
            } else {
                if (nscatt_peel == 0) add(SKG_FULL_DUSDIR, Lextf); else add(SKG_FULL_DUSSCA, Lextf);
            }
        }
    }
    return adds;
}

// Packet flags: bit 0 stellar origin, bit 1 the pending peel-offs follow a scattering, bits 8-15
// the launching stellar component + 1 (0: a dust-emission packet).
SKG_D int pk_comp(const Packet& K) { return ((K.flags >> 8) & 0xff) - 1; }

// Does the group need a traversal?  Frame-only groups skip it when the packet projects off every
// frame (FrameInstrument.cpp:36-37).
SKG_D bool group_needs_traversal(const DevScene& S, int grp, double x, double y, double z) {
    if (!S.group_frame_only[grp]) return true;
    for (int q = S.group_start[grp]; q < S.group_start[grp + 1]; q++)
        if (pixel_on_detector(S.instr[S.group_instr[q]], x, y, z) >= 0) return true;
    return false;
}

struct Launched { double x, y, z, kx, ky, kz, L, Lth; int ok; int stellar; int comp; };
SKG_D int pk_flags(const Launched& o) { return (o.stellar ? 1 : 0) | ((o.comp + 1) << 8); }

// Packet launch: StellarSystem::launch (StellarSystem.cpp:116-158) with the geometry samplers
// (GeometricStellarComp.cpp:75-81), or a dust-emission launch from the cell luminosity CDF
// (PanMonteCarloSimulation.cpp:216-224 self-absorption, :301-323 emission with bias).
__device__ __noinline__ Launched launch_packet(const DevGrid& g, const DevScene& S, int phase, int ell,
                                               uint64_t Npp_total, Philox& rng) {
    Launched o;
    o.ok = 0;
    o.comp = -1;
    const int nl = S.nlambda;
    V3<double> pos, dir;
    if (phase == SKG_PHASE_STELLAR) {
        double Lpp = S.Lv[ell] / (double)Npp_total;
        if (!(Lpp > 0)) return o;
        o.Lth = Lpp / S.min_weight_reduction;
        int N = S.nstellar, h = 0;
        double Lw = Lpp;
        if (N > 1) {
            double eb = S.emission_bias;
            double X = rng.uniform();
            if (X < eb) h = max(0, min(N - 1, (int)(N * X / eb)));
            else h = dlocate_clip(S.Xvv + (size_t)ell * (N + 1), N + 1, (X - eb) / (1.0 - eb));
            double Lh = S.starL[h * nl + ell];
            if (!(Lh > 0)) return o;                         // launched with zero luminosity
            Lw = Lpp * (1.0 / (1.0 - eb + eb * (S.Lv[ell] / N) / Lh));
        }
        pos = geom_position(S.stellar[h], rng);
        dir = iso_direction(rng);
        o.L = Lw; o.stellar = 1; o.comp = h;
    } else {
        double Ltot = S.emit_Ltot[ell];
        if (!(Ltot > 0)) return o;
        double Lem = Ltot / (double)Npp_total;
        o.Lth = Lem / S.min_weight_reduction;
        const int nc = S.ncells;
        const double* cdf = S.emit_cdf + (size_t)ell * (nc + 1);
        double X = rng.uniform(), weight = 1.0;
        int m;
        if (phase == SKG_PHASE_DUST_SELFABS) m = dlocate_clip(cdf, nc + 1, X);
        else {
            double xi = S.dust_emission_bias;
            if (X < xi) m = max(0, min(nc - 1, (int)(nc * X / xi)));
            else m = dlocate_clip(cdf, nc + 1, (X - xi) / (1 - xi));
            weight = 1.0 / (1 - xi + xi * (Ltot / nc) / S.emit_Lv[(size_t)ell * nc + m]);
        }
        o.L = Lem * weight;
        if (!(o.L > 0)) return o;
        pos = random_position_in_cell(g, m, rng);
        dir = iso_direction(rng);
        o.stellar = 0;
    }
    o.x = pos.x; o.y = pos.y; o.z = pos.z; o.kx = dir.x; o.ky = dir.y; o.kz = dir.z;
    o.ok = 1;
    return o;
}

// Peel-off weight toward a direction: the Henyey-Greenstein phase function value
// (DustMix.cpp:648-654), weighted by kappa_sca*rho over the components (:319-331).  A negative
// value aborts the peel-off.
__device__ __noinline__ double peel_weight(const DevScene& S, int ell, int cell, double kx, double ky, double kz,
                                           double gx_, double gy_, double gz_) {
    const int nl = S.nlambda;
    double cosalpha = kx * gx_ + ky * gy_ + kz * gz_;
    if (S.ncomp == 1) {
        double gg = S.asym[ell];
        double t = 1.0 + gg * gg - 2 * gg * cosalpha;
        return (1.0 - gg) * (1.0 + gg) / sqrt(t * t * t);
    }
    double sum = 0, acc = 0;
    for (int h = 0; h < S.ncomp; h++) {
        double wv = (cell >= 0) ? S.ksca[h * nl + ell] * S.rho[(size_t)h * S.ncells + cell] : 0.0;
        double gg = S.asym[h * nl + ell];
        double t = 1.0 + gg * gg - 2 * gg * cosalpha;
        acc += wv * (1.0 - gg) * (1.0 + gg) / sqrt(t * t * t);
        sum += wv;
    }
    return (sum > 0) ? acc / sum : -1.0;
}

// Forced interaction optical depth and weight: MonteCarloSimulation::simulatepropagation
// (:513-531) with Random::exponcutoff (Random.cpp:163-176).  Returns tau; L is reweighted.
#ifndef SKG_SAMPLE_INLINE
#define SKG_SAMPLE_INLINE 0
#endif
#if SKG_SAMPLE_INLINE
SKG_D
#else
__device__ __noinline__
#endif
double sample_interaction(double xi, double taupath, double& L, Philox& rng) {
    auto expcut = [&](double xmax) -> double {
        if (xmax < 1e-10) return rng.uniform() * xmax;
        double x;
        int guard = 0;
        do { x = -log1p(-rng.uniform() * (-expm1(-xmax))); } while (x > xmax && ++guard < 64);
        return fmin(x, xmax);
    };
    if (xi == 0.0) return expcut(taupath);
    double X = rng.uniform();
    double ti = (X < xi) ? rng.uniform() * taupath : expcut(taupath);
    double p = -exp(-ti) / expm1(-taupath);
    double q = (1.0 - xi) * p + xi / taupath;
    L *= p / q;
    return ti;
}

// New direction: DustSystem::randomMixForPosition (DustSystem.cpp:855-869) and the
// Henyey-Greenstein sampling of DustMix::scatteringDirectionAndPolarization (DustMix.cpp:595-602).
__device__ __noinline__ V3<double> scatter_direction(const DevScene& S, int ell, int cell, V3<double> k, Philox& rng) {
    const int nl = S.nlambda;
    int h = 0;
    if (S.ncomp > 1 && cell >= 0) {
        double tot = 0, pv[MAX_COMP];
        for (int c = 0; c < S.ncomp; c++) { pv[c] = S.ksca[c * nl + ell] * S.rho[(size_t)c * S.ncells + cell]; tot += pv[c]; }
        double X = rng.uniform(), acc = 0;
        for (h = 0; h < S.ncomp - 1; h++) { acc += pv[h] / tot; if (X < acc) break; }
    }
    double gg = S.asym[h * nl + ell];
    if (fabs(gg) < 1e-6) return iso_direction(rng);
    double f = ((1.0 - gg) * (1.0 + gg)) / (1.0 - gg + 2.0 * gg * rng.uniform());
    double costheta = (1.0 + gg * gg - f * f) / (2.0 * gg);
    return rotate_direction(k, costheta, rng);
}

// finds the work item of global packet p (items sorted by begin; few items)
SKG_D int find_item(const WorkItem* items, int n, uint64_t p) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (items[mid].begin <= p) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// ---------------------------------------------------------------------------------------------
// event pass

// The direction groups that get a peel-off traversal from (x, y, z), in group order
// (MonteCarloSimulation.cpp:299-357): emission peel-offs carry weight 1, scattering peel-offs the
// phase-function value, and a negative value ends the list (the reference aborts the peel-off).
// With WRITE the jobs are stored from j0 on; returns their number.
template<bool WRITE>
SKG_D int peel_jobs(const DevScene& S, int ell, bool scat, int cell, double kx, double ky, double kz, double x,
                    double y, double z, double L, int p, int j0, int2* jobs, double* jL) {
    int n = 0;
    for (int g = 0; g < S.ngroups; g++) {
        double w = 1.0;
        if (scat) {
            w = peel_weight(S, ell, cell, kx, ky, kz, S.gkx[g], S.gky[g], S.gkz[g]);
            if (w < 0) break;
        }
        if (!group_needs_traversal(S, g, x, y, z)) continue;
        if (WRITE) { jobs[j0 + n] = make_int2(p, g); jL[j0 + n] = L * w; }
        n++;
    }
    return n;
}

constexpr int SED_PRIV = 1024;          // SED bins a block keeps privately (8 KB)

// A packet at its interaction point: propagate, count its scattering peel-offs, scatter
// (simulatepropagation :513-531, peeloffscattering :313-357, simulatescattering :535-543).
template<typename R>
SKG_D void scatter_packet(const RunParams& P, int phase, bool peel_on, Packet& K, int& state, int& npeel, int& nmain,
                          bool& scat_peel, double& kx0, double& ky0, double& kz0, unsigned long long* s_cnt) {
    const WorkItem& It = P.items[K.item];
    const DevScene& S = *P.scenes[It.slot];
    const R si = (R)K.s_int;                        // PhotonPackage::propagate
    K.x = (double)((R)K.x + si * (R)K.kx);
    K.y = (double)((R)K.y + si * (R)K.ky);
    K.z = (double)((R)K.z + si * (R)K.kz);
    // the interaction point lies in the cell of its segment (verified by the stepper)
    if (K.s_int > 0) K.pos_cell = (K.int_cell >= 0) ? K.int_cell : -2;
    kx0 = K.kx; ky0 = K.ky; kz0 = K.kz;
    if (peel_on) {
        scat_peel = true;
        npeel = peel_jobs<false>(S, K.ell, true, K.int_cell, kx0, ky0, kz0, K.x, K.y, K.z, K.L, 0, 0, nullptr, nullptr);
    }
    Philox rng;
    rng.init(It.seed, K.id, (uint32_t)K.ell | ((uint32_t)phase << 24));
    rng.c0 = K.rngc;
    const V3<double> kn = scatter_direction(S, K.ell, K.int_cell, mk3(K.kx, K.ky, K.kz), rng);
    K.rngc = rng.c0;
    K.kx = (double)(R)kn.x; K.ky = (double)(R)kn.y; K.kz = (double)(R)kn.z;
    K.nscatt++;
    atomicAdd(&s_cnt[C_SCATT], 1ull);
    nmain = 1;
    state = PK_WAIT;
}

// Free records take new packets (all lanes of the warp call this; `need` marks the lanes whose
// record is free): one work-counter atomic per warp; a launch with zero luminosity takes the next
// packet; a record finds none once the work counter is past the batch's packets.
template<typename R>
SKG_D void take_packets(const RunParams& P, const BatchHeader& H, int phase, bool peel_on, int lane, bool need,
                        Packet& K, int& state, int& npeel, int& nmain, unsigned long long* s_cnt) {
    const unsigned FULL = 0xffffffffu;
    while (__any_sync(FULL, need)) {
        const unsigned want = __ballot_sync(FULL, need);
        const int leader = __ffs(want) - 1;
        unsigned long long base = 0;
        if (lane == leader) base = atomicAdd(P.work, (unsigned long long)__popc(want));
        base = __shfl_sync(FULL, base, leader);
        if (need) {
            const uint64_t gp = base + __popc(want & ((1u << lane) - 1));
            if (gp >= H.total) {
                state = PK_DONE; need = false;
            } else {
                const int it = find_item(P.items, H.nitems, gp);
                const WorkItem It = P.items[it];
                const uint64_t q = gp - It.begin;
                const int ei = (int)(q / It.count);
                const uint64_t ip = It.first + (q - (uint64_t)ei * It.count);
                const int ell = P.ells[It.ell0 + ei];
                Philox rng;
                rng.init(It.seed, ip, (uint32_t)ell | ((uint32_t)phase << 24));
                atomicAdd(&s_cnt[C_PACKETS], 1ull);
                const DevScene& S = *P.scenes[It.slot];
                const Launched o = launch_packet(P.grids[It.slot], S, phase, ell, It.npp_total, rng);
                if (o.ok) {
                    K.x = (double)(R)o.x; K.y = (double)(R)o.y; K.z = (double)(R)o.z;
                    K.kx = (double)(R)o.kx; K.ky = (double)(R)o.ky; K.kz = (double)(R)o.kz;
                    K.L = o.L; K.Lth = o.Lth; K.s_int = 0;
                    K.id = ip; K.item = it; K.ell = ell; K.nscatt = 0;
                    K.pos_cell = -2; K.int_cell = -1; K.rngc = rng.c0;
                    K.flags = pk_flags(o); K.peel_n = 0;
                    npeel = peel_on ? peel_jobs<false>(S, ell, false, -1, 0, 0, 0, K.x, K.y, K.z, K.L, 0, 0, nullptr,
                                                       nullptr)
                                    : 0;
                    nmain = S.ncomp > 0 ? 1 : 0;            // without dust the life cycle ends here
                    state = nmain ? PK_WAIT : PK_TERM;
                    need = false;
                }
            }
        }
    }
}

// Appends a packet's jobs (all lanes of the warp call this), one reservation per warp for each
// kind: the path jobs (the longest) from index 0, a packet's peel-off jobs contiguous from index
// npool on; counts the packets with work.
SKG_D void append_jobs(const WaveParams& W, int p, Packet& K, int npeel, int nmain, bool scat_peel, double kx0,
                       double ky0, double kz0, int lane) {
    const unsigned FULL = 0xffffffffu;
    int inm = nmain, inp = npeel;
    for (int o = 1; o < 32; o <<= 1) {
        const int tm = __shfl_up_sync(FULL, inm, o), tp = __shfl_up_sync(FULL, inp, o);
        if (lane >= o) { inm += tm; inp += tp; }
    }
    const int totm = __shfl_sync(FULL, inm, 31), totp = __shfl_sync(FULL, inp, 31);
    unsigned bm = 0, bp = 0;
    if (lane == 31) {
        if (totm > 0) bm = atomicAdd(W.jcount, (unsigned)totm);
        if (totp > 0) bp = atomicAdd(W.jcount + 1, (unsigned)totp);
    }
    bm = __shfl_sync(FULL, bm, 31);
    bp = __shfl_sync(FULL, bp, 31);
    const unsigned busy = __ballot_sync(FULL, npeel + nmain > 0);
    if (lane == 0 && busy) {
        atomicAdd(W.jcount + 3, (unsigned)__popc(busy));
        atomicMax(W.last_busy, (unsigned)W.wave);
    }
    if (npeel > 0) {
        const int j0 = W.npool + (int)(bp + inp - npeel);
        const DevScene& S = *W.R.scenes[W.R.items[K.item].slot];
        peel_jobs<true>(S, K.ell, scat_peel, K.int_cell, kx0, ky0, kz0, K.x, K.y, K.z, K.L, p, j0, W.jobs, W.jL);
        K.peel_j0 = j0;
    }
    K.peel_n = npeel;
    if (nmain) W.jobs[bm + inm - 1] = make_int2(p, JOB_MAIN);
}

template<typename R, bool STRIDE>
__global__ void __launch_bounds__(SKG_EVENT_THREADS, SKG_EVENT_MIN_BLOCKS * 256 / SKG_EVENT_THREADS) event_kernel(const WaveParams W) {
    __shared__ unsigned long long s_cnt[C_N];
    __shared__ double s_sed[SED_PRIV];
    const RunParams& P = W.R;
    const BatchHeader H = *P.hdr;
    // a launch of one simulation tallies its SED bins per block and adds them once at the end
    const int sed_bins = (H.nslots == 1) ? P.scenes[0]->sed_bins : 0;
    double* const psed = (sed_bins > 0 && sed_bins <= SED_PRIV) ? s_sed : nullptr;
    if (threadIdx.x < C_N) s_cnt[threadIdx.x] = 0;
    if (psed) for (int t = threadIdx.x; t < sed_bins; t += blockDim.x) s_sed[t] = 0.0;
    __syncthreads();
#if !SKG_LAUNCH_KERNEL
    const int phase = H.phase;
    const bool peel_on = phase != SKG_PHASE_DUST_SELFABS;
#endif
    const int lane = threadIdx.x & 31;
#if SKG_LAUNCH_KERNEL
    const unsigned FULL = 0xffffffffu;
#endif
    // STRIDE: the resident blocks stride over the pool; otherwise one thread per record
#pragma unroll 1
    for (int base = blockIdx.x * blockDim.x, it = 0; STRIDE ? base < W.npool : it == 0;
         base += gridDim.x * blockDim.x, it++) {
    const int p = base + threadIdx.x;

    Packet K;
    int state = PK_DONE;
    if (p < W.npool) { K = W.pk[p]; state = K.state; }
    const bool was_live = state != PK_DONE;
    if (state == PK_WAIT) {                       // a path job that was not walked: drop the packet
        atomicOr(P.err, ERR_CAPACITY); atomicAdd(&s_cnt[C_ERR], 1ull); state = PK_TERM;
    }

    // 1. the peel-offs walked in the previous wave (Instrument::detect of every group member)
    if (was_live && K.peel_n > 0) {
        const DevScene& S = *P.scenes[P.items[K.item].slot];
        const int nsp = (K.flags & 2) ? K.nscatt : 0;   // the peel-off copy counts the scattering
        int pix = 0;
        for (int i = 0; i < K.peel_n; i++) {
            const int j = K.peel_j0 + i;
            pix += detect_group(S, W.pjobs[j].y, K.ell, W.pjL[j], W.pjtau[j], nsp, (K.flags & 1) != 0,
                                pk_comp(K), K.x, K.y, K.z, psed);
        }
        atomicAdd(&s_cnt[C_PIX], (unsigned long long)pix);
        atomicAdd(&s_cnt[C_PEEL], (unsigned long long)K.peel_n);
        K.peel_n = 0;
    }

    // 2. a packet at its interaction point: propagate, count its scattering peel-offs, scatter
    int npeel = 0, nmain = 0;
    bool scat_peel = false;
    double kx0 = 0, ky0 = 0, kz0 = 0;              // direction before the scattering
#if SKG_LAUNCH_KERNEL
    // (in the launch pass, with every lane of its warps scattering)
    {
        const bool inter = p < W.npool && state == PK_INTERACT;
        const unsigned im = __ballot_sync(FULL, inter);
        if (im) {
            const int leader = __ffs(im) - 1;
            unsigned base = 0;
            if (lane == leader) base = atomicAdd(W.jcount + 6, (unsigned)__popc(im));
            base = __shfl_sync(FULL, base, leader);
            if (inter) W.intlist[base + __popc(im & ((1u << lane) - 1))] = p;
        }
    }
#else
    if (state == PK_INTERACT)
        scatter_packet<R>(P, phase, peel_on, K, state, npeel, nmain, scat_peel, kx0, ky0, kz0, s_cnt);
#endif

#if SKG_LAUNCH_KERNEL
    // 3. free records go on the wave's free list: the launch pass gives them new packets, every
    //    lane of its warps launching (here a warp's launches would run beside its scatterings)
    {
        const bool freed = p < W.npool && (state == PK_EMPTY || state == PK_TERM);
        const unsigned fm = __ballot_sync(FULL, freed);
        if (fm) {
            const int leader = __ffs(fm) - 1;
            unsigned base = 0;
            if (lane == leader) base = atomicAdd(W.jcount + 5, (unsigned)__popc(fm));
            base = __shfl_sync(FULL, base, leader);
            if (freed) W.freelist[base + __popc(fm & ((1u << lane) - 1))] = p;
        }
    }
#else
    // 3. free records take new packets
    take_packets<R>(P, H, phase, peel_on, lane, state == PK_EMPTY || state == PK_TERM, K, state, npeel, nmain, s_cnt);
#endif

#if SKG_LAUNCH_KERNEL
    // every live record is now on one of the two lists, and the scatter-and-launch pass rewrites
    // it (jobs, state, the cleared peel-off count): this pass only read it
    (void)npeel; (void)nmain; (void)scat_peel; (void)kx0; (void)ky0; (void)kz0; (void)was_live;
#else
    // 4. append the jobs
    append_jobs(W, p, K, npeel, nmain, scat_peel, kx0, ky0, kz0, lane);
    if (p < W.npool && was_live) {
        K.flags = (K.flags & ~2) | (scat_peel ? 2 : 0);
        K.state = state;
        W.pk[p] = K;
    }
#endif
    }   // records of this block
    __syncthreads();
    if (threadIdx.x < C_N && s_cnt[threadIdx.x]) atomicAdd(P.counters + threadIdx.x, s_cnt[threadIdx.x]);
    if (psed) {
        const DevScene& S0 = *P.scenes[0];
        for (int t = threadIdx.x; t < sed_bins; t += blockDim.x) {
            const double v = s_sed[t];
            if (v == 0.0) continue;
            int i = 0;
            while (i + 1 < S0.ninstr && S0.sed_base[i + 1] <= t) i++;
            atomicAdd(S0.instr[i].sed + (t - S0.sed_base[i]), v);
        }
    }
}

// Scatter-and-launch pass: one thread per record the event pass found at its interaction point
// (propagation, scattering peel-offs, scattering), then one per record it freed (StellarSystem::launch
// and the samplers, or the dust-emission launch), every lane of a warp doing the same work; the
// packets' jobs are appended as the event pass does.
template<typename R>
__global__ void __launch_bounds__(SKG_EVENT_THREADS) launch_kernel(const WaveParams W) {
    __shared__ unsigned long long s_cnt[C_N];
    const RunParams& P = W.R;
    const BatchHeader H = *P.hdr;
    if (threadIdx.x < C_N) s_cnt[threadIdx.x] = 0;
    __syncthreads();
    const int phase = H.phase;
    const bool peel_on = phase != SKG_PHASE_DUST_SELFABS;
    const int lane = threadIdx.x & 31;
    const unsigned nint = W.jcount[6];
    for (unsigned b0 = blockIdx.x * blockDim.x; b0 < nint; b0 += gridDim.x * blockDim.x) {
        const unsigned i = b0 + threadIdx.x;
        const bool mine = i < nint;
        const int p = mine ? W.intlist[i] : 0;
        Packet K;
        int state = PK_DONE, npeel = 0, nmain = 0;
        bool scat_peel = false;
        double kx0 = 0, ky0 = 0, kz0 = 0;
        if (mine) {
            K = W.pk[p];
            state = K.state;
            scatter_packet<R>(P, phase, peel_on, K, state, npeel, nmain, scat_peel, kx0, ky0, kz0, s_cnt);
        }
        append_jobs(W, p, K, npeel, nmain, scat_peel, kx0, ky0, kz0, lane);
        if (mine) {
            K.flags = (K.flags & ~2) | (scat_peel ? 2 : 0);   // the pending peel-offs follow a scattering
            K.state = state;
            W.pk[p] = K;
        }
    }
    const unsigned nfree = W.jcount[5];
    for (unsigned b0 = blockIdx.x * blockDim.x; b0 < nfree; b0 += gridDim.x * blockDim.x) {
        const unsigned i = b0 + threadIdx.x;
        const bool mine = i < nfree;
        const int p = mine ? W.freelist[i] : 0;
        Packet K;
        int state = PK_DONE, npeel = 0, nmain = 0;
        if (mine) { K = W.pk[p]; state = K.state; }
        take_packets<R>(P, H, phase, peel_on, lane, mine, K, state, npeel, nmain, s_cnt);
        append_jobs(W, p, K, npeel, nmain, false, 0, 0, 0, lane);
        if (mine) {
            K.flags &= ~2;
            K.state = state;
            W.pk[p] = K;
        }
    }
    __syncthreads();
    if (threadIdx.x < C_N && s_cnt[threadIdx.x]) atomicAdd(P.counters + threadIdx.x, s_cnt[threadIdx.x]);
}

// ---------------------------------------------------------------------------------------------
// traversal pass

// Absorption in cell m of a path step: simulateescapeandabsorption (MonteCarloSimulation.cpp:441-462)
// with OligoDustSystem::absorb / PanDustSystem::absorb.  The tables are wavelength-major on the
// device ([ell][m]): a wave carries the packets of one or two wavelengths (packets are handed out
// wavelength by wavelength), so its tallies fall in one slice of the table that stays in L2.  v1 = L e^-tau on entry (a running product,
// one expm1 per absorbing step: L e^-tau (1 - e^-dtau) = -v1 expm1(-dtau)); v2 accumulates L_sca with
// the local albedo when there are several dust components.  Returns 1 when a tally was stored.
template<typename R>
SKG_D int absorb_step(const DevScene& S, int phase, int m, int ell, double dtau, double& v1, double& v2) {
    if (m < 0) return 0;
    const bool store = (phase == SKG_PHASE_STELLAR) ? (S.store_abs != 0) : (phase == SKG_PHASE_DUST_SELFABS);
    double* labs = (phase == SKG_PHASE_STELLAR) ? S.labs_stel : S.labs_dust;
    if (S.ncomp == 1) {
        if (!store) return 0;
        const double em = expm1(-dtau);
        const double Lintm = -v1 * em;
        v1 += v1 * em;
        atomicAdd(labs + (size_t)ell * S.ncells + m, (1.0 - S.albedo[ell]) * Lintm);
        return 1;
    }
    double ksca = 0, kext = 0;
    for (int h = 0; h < S.ncomp; h++) {
        const double rh = rho_load<R>(S, (size_t)h * S.ncells + m);
        ksca += rh * S.ksca[h * S.nlambda + ell]; kext += rh * S.kext[h * S.nlambda + ell];
    }
    const double alb = (kext > 0.0) ? ksca / kext : 0.0;
    const double em = expm1(-dtau);
    const double Lintm = -v1 * em;
    v1 += v1 * em;
    v2 += alb * Lintm;
    if (!store) return 0;
    atomicAdd(labs + (size_t)ell * S.ncells + m, (1.0 - alb) * Lintm);
    return 1;
}

// End of the packet's own path (simulateescapeandabsorption :441-462, the termination test of
// dostellaremissionchunk :283, simulatepropagation :513-531).  Returns 1 when the path must be
// re-walked to tau_int (the packet's luminosity is then already in its record), 0 when the packet
// record is complete, -1 on an error.  Inlined: as a call
// it made the traversal kernel keep a 264-byte stack frame for the call's saved registers (88
// bytes inlined; the traversal pass ran 11 % faster).
SKG_D int after_path(const WaveParams& W, const DevScene& S, int p, int phase, int ell,
                     double taupath, double Lsca, double& L, double& tau_int) {
    Packet& K = W.pk[p];
    if (taupath < 0.0 || isnan(taupath) || isinf(taupath)) {   // DustSystem.cpp:953-955
        atomicOr(W.R.err, ERR_NAN_TAU);
        K.state = PK_TERM;
        return -1;
    }
    if (S.ncomp == 1) L = L * S.albedo[ell] * (-expm1(-taupath));
    else L = Lsca;
    if (L <= 0 || (L <= K.Lth && K.nscatt >= S.min_scatt_events)) { K.state = PK_TERM; return 0; }
    if (K.nscatt >= W.R.max_scatt) {
        atomicOr(W.R.err, ERR_SCATT_BUDGET);
        K.state = PK_TERM;
        return -1;
    }
    if (taupath == 0.0) {                 // no dust ahead: scatter where the packet is
        K.L = L; K.s_int = 0; K.int_cell = K.pos_cell >= 0 ? K.pos_cell : -1; K.state = PK_INTERACT;
        return 0;
    }
    const WorkItem& It = W.R.items[K.item];
    Philox rng;
    rng.init(It.seed, K.id, (uint32_t)ell | ((uint32_t)phase << 24));
    rng.c0 = K.rngc;
    tau_int = sample_interaction(S.xi, taupath, L, rng);
    K.rngc = rng.c0;
    K.L = L;                              // the weight the packet carries to its interaction point
    return 1;
}

// A checkpoint of packet p's path walk (slot i): the stepper's state, then the optical depth and
// the path length walked (from the packet's position) and the step count.
template<class St>
SKG_D void save_ckpt(const WaveParams& W, int p, int i, const St& st, double tau) {
    const Packet& K = W.pk[p];
    const float s = st.walked_from((float)K.x, (float)K.y, (float)K.z);
    float4* c = W.ckpt + ((size_t)p * SKG_CKPT_N + i) * 2;
    c[0] = st.ckpt();
    c[1] = make_float4(__int_as_float(__double2loint(tau)), __int_as_float(__double2hiint(tau)), s,
                       __int_as_float(st.steps));
}

// Resumes the re-walk of packet p's path toward tau_int at its last checkpoint (of nck) whose
// optical depth is at most tau_int: the steps before it would not have reached tau_int.  Returns
// false when there is none (the re-walk starts at the path's start).
template<class St>
SKG_D bool resume_ckpt(const WaveParams& W, const DevGrid& g, int p, int nck, double tau_int, St& st, double& tau,
                       double& s) {
    const float4* c = W.ckpt + (size_t)p * SKG_CKPT_N * 2;
    int lo = -1, hi = nck - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        const float4 b = c[2 * mid + 1];
        if (__hiloint2double(__float_as_int(b.y), __float_as_int(b.x)) <= tau_int) lo = mid; else hi = mid - 1;
    }
    if (lo < 0) return false;
    const float4 b = c[2 * lo + 1];
    const Packet& K = W.pk[p];
    st.resume(g, (float)K.x, (float)K.y, (float)K.z, (float)K.kx, (float)K.ky, (float)K.kz, K.pos_cell, c[2 * lo],
              __float_as_int(b.w));
    tau = __hiloint2double(__float_as_int(b.y), __float_as_int(b.x));
    s = (double)b.z;
    return true;
}

// MODE: 0 every job of the wave; 1 the path jobs only; 2 the peel-off jobs only (a lean
// instantiation: optical depth alone, no path state)
// Resident blocks per SM of each instantiation.  The Voronoi path-job kernel runs at 3 blocks (80
// registers, no spills: its neighbour scan keeps more state): 1219 against 1273 ms per 10^7-packet
// phase; the tree and Cartesian ones are faster at 4 (189 against 194 ms, 94 against 100 ms).
template<int MODE, template<typename> class Stepper> struct TravBlocks { static constexpr int value = SKG_TRAV_MIN_BLOCKS; };
template<template<typename> class Stepper> struct TravBlocks<1, Stepper> { static constexpr int value = SKG_PATH_MIN_BLOCKS; };
template<> struct TravBlocks<1, VoronoiStepper> { static constexpr int value = SKG_VOR_PATH_MIN_BLOCKS; };
template<template<typename> class Stepper> struct TravBlocks<2, Stepper> { static constexpr int value = SKG_PEEL_MIN_BLOCKS; };

template<typename R, template<typename> class Stepper, int MODE, bool ONE>
__global__ void __launch_bounds__(256, (TravBlocks<MODE, Stepper>::value)) trav_kernel(const WaveParams W) {
    extern __shared__ unsigned char smem_raw[];
    DevGrid* sg = reinterpret_cast<DevGrid*>(smem_raw);
    // the grid of a job's slot: a single-simulation launch (ONE) reads it from the kernel's
    // parameters, whose fields are constant-bank operands; a batch from the block's shared copy,
    // which the compiler reloads after the shared-memory counter atomics of the loop
    auto grid_of = [&](int sl) -> const DevGrid& {
        if constexpr (ONE) return W.g0; else return sg[sl];
    };
    __shared__ const DevScene* s_scene[MAX_SLOTS];
    __shared__ unsigned long long s_cnt[C_N];
    const RunParams& P = W.R;
    const BatchHeader H = *P.hdr;
    for (int i = threadIdx.x; i < C_N; i += blockDim.x) s_cnt[i] = 0;
    for (int i = threadIdx.x; i < H.nslots; i += blockDim.x) { sg[i] = P.grids[i]; s_scene[i] = P.scenes[i]; }
    __syncthreads();
#if SKG_PDL
    // the path-job kernel lets the peel-off-job kernel of the same wave be scheduled now: its blocks
    // become resident as this kernel's blocks run out of jobs and exit, so the two overlap in the
    // tail of this one.  The peel-off kernel reads only what the event pass wrote (complete before
    // this kernel started); the one word both may touch, a packet's start cell, is written here
    // only from "unknown" to the cell, and either value is a valid hint for the peel-off walk.
    if (MODE == 1) asm volatile("griddepcontrol.launch_dependents;");
#endif
    const unsigned nmainj = W.jcount[0];
    const unsigned njobs = MODE == 0 ? nmainj + W.jcount[1] : MODE == 1 ? nmainj : W.jcount[1];
    unsigned* const taken = W.jcount + (MODE == 2 ? 4 : 2);
    const int phase = H.phase;
    const int lane = threadIdx.x & 31;
    const int refill_lanes = P.refill > 0 ? P.refill : (MODE == 2 ? SKG_REFILL_PEEL : SKG_REFILL_LANES);

    int j = -1;                       // the lane's job (-1: none)
    int p = 0, slot = 0, ell = 0;
    int kind = 0;                     // 0 peel-off, 1 path, 2 re-walk to the interaction point
    double tau = 0;                   // optical depth walked
    // values of one job kind share two registers -- path: v1 = L e^-tau (the luminosity that
    // reaches the current cell, kept as a running product: one expm1 per absorbing cell step),
    // v2 = L_sca (several dust components); re-walk: v1 = path length walked, v2 = the
    // interaction optical depth
    double v1 = 0, v2 = 0;
    float kext1 = -1.f;               // kappa_ext at the job's wavelength (one dust component), else -1
    unsigned c_steps = 0;
    Stepper<R> st;
    constexpr bool CKPT = SKG_CKPT && MODE != 2 && Resumable<Stepper<R>>::value;
    int nck = 0;                      // checkpoints of the path walk

    while (true) {
        // lanes without a job take the next ones: one atomic per warp
        const unsigned live = __activemask();
        const bool need = j < 0;
        const unsigned want = __ballot_sync(live, need);
        // lanes whose path walk ended (kind 3) run the end of the path together
        const unsigned pend = (MODE == 2) ? 0u : __ballot_sync(live, kind == 3);
        const bool idle = (live & ~want & ~pend) == 0;      // no lane of the warp is walking
        if (pend && (__popc(pend) >= SKG_AFTER_LANES || idle)) {
            if (kind == 3) {
                const DevGrid& g = grid_of(slot);
                const DevScene& S = *s_scene[slot];
                double L = W.pk[p].L, tau_int = 0;      // the packet's luminosity at the path start
                const int rc = after_path(W, S, p, phase, ell, tau, v2, L, tau_int);
                if (rc == 1) {
                    kind = 2; v2 = tau_int;
                    bool resumed = false;
                    if constexpr (CKPT) resumed = W.ckpt && resume_ckpt(W, g, p, nck, tau_int, st, tau, v1);
                    if (!resumed) {
                        const Packet& K = W.pk[p];
                        st.init(g, (R)K.x, (R)K.y, (R)K.z, (R)K.kx, (R)K.ky, (R)K.kz, K.pos_cell);
                        tau = 0; v1 = 0;
                        R d0;
                        while (st.pd.pop(d0)) v1 += (double)d0;
                    }
                } else {
                    if (rc < 0) atomicAdd(&s_cnt[C_ERR], 1ull);
                    j = -1;
                    kind = 0;
                }
            }
            continue;
        }
        if (want && (__popc(want) >= refill_lanes || (live & ~want & ~pend) == 0)) {
            const int leader = __ffs(want) - 1;
            unsigned base = 0;
            if (lane == leader) base = atomicAdd(taken, (unsigned)__popc(want));
            base = __shfl_sync(live, base, leader);
            if (need) {
                const unsigned jj = base + __popc(want & ((1u << lane) - 1));
                if (jj >= njobs) break;
                if (MODE == 0) j = jj < nmainj ? (int)jj : W.npool + (int)(jj - nmainj);
                else if (MODE == 1) j = (int)jj;
                else j = W.npool + (int)jj;
                const int2 jb = W.jobs[j];
                p = jb.x;
                const Packet& K = W.pk[p];
                ell = K.ell;
                slot = P.items[K.item].slot;
                const DevScene& S = *s_scene[slot];
                const int hint = K.pos_cell;
                kext1 = (S.ncomp == 1) ? (float)S.kext[ell] : -1.f;
                R kx, ky, kz;
                if (MODE != 2 && jb.y == JOB_MAIN) { kx = (R)K.kx; ky = (R)K.ky; kz = (R)K.kz; kind = 1; v1 = K.L; v2 = 0; nck = 0; }
                else { kx = (R)S.gkx[jb.y]; ky = (R)S.gky[jb.y]; kz = (R)S.gkz[jb.y]; kind = 0; }
                st.init(grid_of(slot), (R)K.x, (R)K.y, (R)K.z, kx, ky, kz, hint);
                if (kind == 1 && hint == -2) W.pk[p].pos_cell = st.cell0;
                tau = 0;
                // entry segments outside the grid (m = -1) carry no optical depth: only the
                // re-walk, which measures length, takes them
            }
        }

        if (j < 0 || kind == 3) continue;   // waiting for enough lanes to refill / end paths together

        const DevGrid& g = grid_of(slot);
        const DevScene& S = *s_scene[slot];
        // one cell step of the job (m, ds, its optical depth); true when it ended the job (a re-walk
        // that reached the interaction optical depth)
        auto take_step = [&](int m, R ds, double dtau) -> bool {
            c_steps++;
            if (kind == 0) {
                tau += dtau;
            } else if (kind == 1) {
                if (absorb_step<R>(S, phase, m, ell, dtau, v1, v2)) atomicAdd(&s_cnt[C_ABS], 1ull);
                tau += dtau;
                if constexpr (CKPT) {
                    if (W.ckpt && nck < SKG_CKPT_N && st.steps >= (nck + 1) * SKG_CKPT_STRIDE && !st.done) {
                        save_ckpt(W, p, nck, st, tau);
                        nck++;
                    }
                }
            } else {
                const double tn = tau + dtau, sn = v1 + (double)ds;
                if (tn > v2) {
                    Packet& K = W.pk[p];
                    K.s_int = v1 + ((v2 - tau) / (tn - tau)) * (sn - v1);
                    K.int_cell = m;
                    K.state = PK_INTERACT;
                    atomicAdd(&s_cnt[C_TRAV], 1ull);
                    atomicAdd(&s_cnt[C_NBR], (unsigned long long)st.nscanned());
                    atomicAdd(&s_cnt[C_FB], (unsigned long long)st.fallbacks);
                    j = -1;
                    return true;
                }
                tau = tn; v1 = sn;
            }
            return false;
        };
        // the traversal reached the edge of the grid
        auto at_edge = [&]() {
            atomicAdd(&s_cnt[C_TRAV], 1ull);
            atomicAdd(&s_cnt[C_NBR], (unsigned long long)st.nscanned());
            atomicAdd(&s_cnt[C_FB], (unsigned long long)st.fallbacks);
            if (st.steps > g.max_steps) { atomicOr(P.err, ERR_STEP_BUDGET); atomicAdd(&s_cnt[C_ERR], 1ull); }
            if (kind == 0) {
                W.jtau[j] = tau;
                j = -1;
            } else if (kind == 1) {
                kind = 3;                       // the end of the path runs with other lanes' (above)
            } else {
                // DustGridPath::pathlength: an optical depth beyond the last segment gives the full length
                Packet& K = W.pk[p];
                K.s_int = v1; K.int_cell = -1; K.state = PK_INTERACT;
                j = -1;
            }
        };

        // cell steps: up to SKG_INNER_STEPS of them before the warp looks at refills again.  (Walking
        // four steps ahead and loading their densities together, for the walks whose records do
        // not carry the density, was slower: Cartesian traversal pass 83 against 64 ms, Voronoi
        // peel-off walks 298 against 258 ms; the walk is issue-bound, not waiting on those loads.)
#pragma unroll 1
        for (int is = 0; is < (MODE == 2 ? SKG_INNER_STEPS : SKG_INNER_PATH); is++) {
            int m; R ds;
            if (st.walk(g, m, ds)) {
                // one dust component: the FP32 tree walk carries the cell density in its leaf record
                if (take_step(m, ds, step_dtau<R>(S, st, kext1, m, ell, ds))) break;
            } else {
                at_edge();
                break;
            }
        }
    }

    atomicAdd(&s_cnt[C_STEPS], (unsigned long long)c_steps);
    __syncthreads();
    if (threadIdx.x < C_N && s_cnt[threadIdx.x]) atomicAdd(P.counters + threadIdx.x, s_cnt[threadIdx.x]);
#if SKG_PDL
    // the peel-off kernel completes only after the path-job kernel it overlapped (and its writes
    // are visible), so the next wave's event pass, ordered after this kernel, sees both
    if (MODE == 2) asm volatile("griddepcontrol.wait;" ::: "memory");
#endif
}

// ---------------------------------------------------------------------------------------------
// tail pass: the end of a phase
//
// When few packets are left in flight, each wave costs about as long as its longest walk while
// most of the device idles, and a packet still needs a wave per event.  The tail pass gives every
// remaining packet a thread that runs the rest of its life at once -- the previous wave's pending
// peel-off detections, then interaction, scattering peel-offs, scattering, path and re-walk until
// it terminates, then further packets while the work counter has any -- with the same random
// streams, samplers and tallies as the waves (device functions shared with the event and traversal
// passes), so a phase gives the same results with or without it, up to the summation order of the
// FP64 tally atomics.

// Optical depth from (x, y, z) toward (kx, ky, kz) to the edge of the grid (DustSystem::opticaldepth,
// DustSystem.cpp:960-976).
template<typename R, template<typename> class Stepper>
SKG_D double tail_tau(const DevGrid& g, const DevScene& S, int ell, R x, R y, R z, R kx, R ky, R kz, int hint,
                      unsigned long long* cnt, unsigned* err) {
    Stepper<R> st;
    st.init(g, x, y, z, kx, ky, kz, hint);
    const float kext1 = (S.ncomp == 1) ? (float)S.kext[ell] : -1.f;
    double tau = 0;
    int m; R ds;
    while (st.walk(g, m, ds)) {
        cnt[C_STEPS]++;
        tau += step_dtau<R>(S, st, kext1, m, ell, ds);
    }
    cnt[C_TRAV]++; cnt[C_NBR] += st.nscanned(); cnt[C_FB] += st.fallbacks;
    if (st.steps > g.max_steps) { atomicOr(err, ERR_STEP_BUDGET); cnt[C_ERR]++; }
    return tau;
}

// The peel-offs of the packet from its position (peeloffemission :299-309, peeloffscattering
// :313-357): one traversal per direction group that needs one, detected at once.  nsp: the
// scattering count the peel-off copy carries (0 for emission).
template<typename R, template<typename> class Stepper>
SKG_D void tail_peel(const DevGrid& g, const DevScene& S, const Packet& K, bool scat, int nsp, double kx0,
                     double ky0, double kz0, unsigned long long* cnt, unsigned* err) {
    for (int grp = 0; grp < S.ngroups; grp++) {
        double w = 1.0;
        if (scat) {
            w = peel_weight(S, K.ell, K.int_cell, kx0, ky0, kz0, S.gkx[grp], S.gky[grp], S.gkz[grp]);
            if (w < 0) break;
        }
        if (!group_needs_traversal(S, grp, K.x, K.y, K.z)) continue;
        const double tau = tail_tau<R, Stepper>(g, S, K.ell, (R)K.x, (R)K.y, (R)K.z, (R)S.gkx[grp], (R)S.gky[grp],
                                                (R)S.gkz[grp], K.pos_cell, cnt, err);
        cnt[C_PEEL]++;
        cnt[C_PIX] += detect_group(S, grp, K.ell, K.L * w, tau, nsp, (K.flags & 1) != 0, pk_comp(K), K.x, K.y, K.z,
                                   nullptr);
    }
}

// The packet's own path and, when it interacts, the re-walk to the interaction point: the path job
// of the traversal pass.  Leaves the record in PK_INTERACT or PK_TERM.
template<typename R, template<typename> class Stepper>
SKG_D void tail_path(const WaveParams& W, const DevGrid& g, const DevScene& S, int p, int phase,
                     unsigned long long* cnt) {
    Packet& K = W.pk[p];
    const int ell = K.ell;
    const float kext1 = (S.ncomp == 1) ? (float)S.kext[ell] : -1.f;
    Stepper<R> st;
    const int hint = K.pos_cell;
    st.init(g, (R)K.x, (R)K.y, (R)K.z, (R)K.kx, (R)K.ky, (R)K.kz, hint);
    if (hint == -2) K.pos_cell = st.cell0;
    double tau = 0, v1 = K.L, v2 = 0;
    constexpr bool CKPT = SKG_CKPT && Resumable<Stepper<R>>::value;
    int nck = 0;                                  // checkpoints, as the traversal pass takes them
    int m; R ds;
    while (st.walk(g, m, ds)) {
        cnt[C_STEPS]++;
        const double dtau = step_dtau<R>(S, st, kext1, m, ell, ds);
        cnt[C_ABS] += absorb_step<R>(S, phase, m, ell, dtau, v1, v2);
        tau += dtau;
        if constexpr (CKPT) {
            if (W.ckpt && nck < SKG_CKPT_N && st.steps >= (nck + 1) * SKG_CKPT_STRIDE && !st.done) {
                save_ckpt(W, p, nck, st, tau);
                nck++;
            }
        }
    }
    cnt[C_TRAV]++; cnt[C_NBR] += st.nscanned(); cnt[C_FB] += st.fallbacks;
    if (st.steps > g.max_steps) { atomicOr(W.R.err, ERR_STEP_BUDGET); cnt[C_ERR]++; }
    double L = K.L, tau_int = 0;
    const int rc = after_path(W, S, p, phase, ell, tau, v2, L, tau_int);
    if (rc < 0) cnt[C_ERR]++;
    if (rc != 1) return;
    // DustGridPath::pathlength on the re-walked path
    double s = 0;
    bool resumed = false;
    if constexpr (CKPT) resumed = W.ckpt && resume_ckpt(W, g, p, nck, tau_int, st, tau, s);
    if (!resumed) {
        st.init(g, (R)K.x, (R)K.y, (R)K.z, (R)K.kx, (R)K.ky, (R)K.kz, K.pos_cell);
        R d0;
        while (st.pd.pop(d0)) s += (double)d0;
        tau = 0;
    }
    while (st.walk(g, m, ds)) {
        cnt[C_STEPS]++;
        const double tn = tau + step_dtau<R>(S, st, kext1, m, ell, ds), sn = s + (double)ds;
        if (tn > tau_int) {
            K.s_int = s + ((tau_int - tau) / (tn - tau)) * (sn - s);
            K.int_cell = m;
            K.state = PK_INTERACT;
            cnt[C_TRAV]++; cnt[C_NBR] += st.nscanned(); cnt[C_FB] += st.fallbacks;
            return;
        }
        tau = tn; s = sn;
    }
    cnt[C_TRAV]++; cnt[C_NBR] += st.nscanned(); cnt[C_FB] += st.fallbacks;
    if (st.steps > g.max_steps) { atomicOr(W.R.err, ERR_STEP_BUDGET); cnt[C_ERR]++; }
    K.s_int = s; K.int_cell = -1; K.state = PK_INTERACT;
}

template<typename R, template<typename> class Stepper>
__global__ void __launch_bounds__(128) tail_kernel(const WaveParams W) {
    const RunParams& P = W.R;
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= W.npool) return;
    Packet& K = W.pk[p];
    int state = K.state;
    if (state == PK_DONE) return;
    const BatchHeader H = *P.hdr;
    const int phase = H.phase;
    const bool peel_on = phase != SKG_PHASE_DUST_SELFABS;
    unsigned long long cnt[C_N];
    for (int c = 0; c < C_N; c++) cnt[c] = 0;
    if (state == PK_WAIT) {                       // a path job that was not walked (as the event pass)
        atomicOr(P.err, ERR_CAPACITY); cnt[C_ERR]++; state = PK_TERM;
    }
    // the peel-offs walked in the last wave
    if (K.peel_n > 0) {
        const DevScene& S = *P.scenes[P.items[K.item].slot];
        const int nsp = (K.flags & 2) ? K.nscatt : 0;
        for (int i = 0; i < K.peel_n; i++) {
            const int j = K.peel_j0 + i;
            cnt[C_PIX] += detect_group(S, W.pjobs[j].y, K.ell, W.pjL[j], W.pjtau[j], nsp, (K.flags & 1) != 0,
                                       pk_comp(K), K.x, K.y, K.z, nullptr);
        }
        cnt[C_PEEL] += K.peel_n;
        K.peel_n = 0;
    }
    while (true) {
        if (state == PK_INTERACT) {
            const WorkItem& It = P.items[K.item];
            const DevScene& S = *P.scenes[It.slot];
            const DevGrid& g = P.grids[It.slot];
            const R si = (R)K.s_int;                // PhotonPackage::propagate
            K.x = (double)((R)K.x + si * (R)K.kx);
            K.y = (double)((R)K.y + si * (R)K.ky);
            K.z = (double)((R)K.z + si * (R)K.kz);
            if (K.s_int > 0) K.pos_cell = (K.int_cell >= 0) ? K.int_cell : -2;
            const double kx0 = K.kx, ky0 = K.ky, kz0 = K.kz;
            if (peel_on) tail_peel<R, Stepper>(g, S, K, true, K.nscatt + 1, kx0, ky0, kz0, cnt, P.err);
            Philox rng;
            rng.init(It.seed, K.id, (uint32_t)K.ell | ((uint32_t)phase << 24));
            rng.c0 = K.rngc;
            const V3<double> kn = scatter_direction(S, K.ell, K.int_cell, mk3(K.kx, K.ky, K.kz), rng);
            K.rngc = rng.c0;
            K.kx = (double)(R)kn.x; K.ky = (double)(R)kn.y; K.kz = (double)(R)kn.z;
            K.nscatt++;
            cnt[C_SCATT]++;
            state = PK_WAIT;
        }
        if (state == PK_WAIT) {
            const int slot = P.items[K.item].slot;
            tail_path<R, Stepper>(W, P.grids[slot], *P.scenes[slot], p, phase, cnt);
            state = K.state;
            continue;
        }
        // a free record takes the next packet while there is one
        const unsigned long long gp = atomicAdd(P.work, 1ull);
        if (gp >= H.total) break;
        const int it = find_item(P.items, H.nitems, gp);
        const WorkItem It = P.items[it];
        const uint64_t q = gp - It.begin;
        const int ei = (int)(q / It.count);
        const uint64_t ip = It.first + (q - (uint64_t)ei * It.count);
        const int ell = P.ells[It.ell0 + ei];
        Philox rng;
        rng.init(It.seed, ip, (uint32_t)ell | ((uint32_t)phase << 24));
        cnt[C_PACKETS]++;
        const DevScene& S = *P.scenes[It.slot];
        const Launched o = launch_packet(P.grids[It.slot], S, phase, ell, It.npp_total, rng);
        state = PK_TERM;
        if (!o.ok) continue;
        K.x = (double)(R)o.x; K.y = (double)(R)o.y; K.z = (double)(R)o.z;
        K.kx = (double)(R)o.kx; K.ky = (double)(R)o.ky; K.kz = (double)(R)o.kz;
        K.L = o.L; K.Lth = o.Lth; K.s_int = 0;
        K.id = ip; K.item = it; K.ell = ell; K.nscatt = 0;
        K.pos_cell = -2; K.int_cell = -1; K.rngc = rng.c0;
        K.flags = pk_flags(o); K.peel_n = 0;
        if (peel_on) tail_peel<R, Stepper>(P.grids[It.slot], S, K, false, 0, 0, 0, 0, cnt, P.err);
        state = S.ncomp > 0 ? PK_WAIT : PK_TERM;   // without dust the life cycle ends here
    }
    K.state = PK_DONE;
    for (int c = 0; c < C_N; c++) if (cnt[c]) atomicAdd(P.counters + c, cnt[c]);
}

// ---------------------------------------------------------------------------------------------
// host side

namespace {

// Resident blocks of a traversal instantiation (persistent grid = this many blocks per SM x SMs).
template<typename R, template<typename> class Stepper, int MODE, bool ONE>
int resident_blocks(size_t smem) {
    static int per = 0, sms = 0;
    if (per == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, trav_kernel<R, Stepper, MODE, ONE>, 256, smem);
        if (per <= 0) per = 1;
    }
    return sms * per;
}

template<typename R, template<typename> class Stepper, bool ONE>
cudaError_t enqueue_wave(const WaveParams& W, int nslots, int trav_blocks, cudaEvent_t mid, cudaStream_t s) {
    const size_t smem = (size_t)nslots * sizeof(DevGrid);
    const int need = (W.npool + SKG_EVENT_THREADS - 1) / SKG_EVENT_THREADS;
    // (Cartesian grids only: the octree's event pass, detections into three 512^2 frames, is slower
    // strided at any pool size -- 2^21: 52.2 against 44.8 ms over 150 launches -- its heavier
    // records unevenly spread over the resident blocks)
    constexpr bool cart = std::is_same<Stepper<R>, CartStepper<R>>::value || std::is_same<Stepper<R>, CartUniStepper<R>>::value;
    if (cart && W.npool <= SKG_EVENT_STRIDE_POOL) {
        static int esms = 0, eper = 1;
        if (esms == 0) {
            int dev = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&esms, cudaDevAttrMultiProcessorCount, dev);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&eper, event_kernel<R, true>, SKG_EVENT_THREADS, 0);
            if (eper <= 0) eper = 1;
        }
        event_kernel<R, true><<<std::min(need, esms * eper), SKG_EVENT_THREADS, 0, s>>>(W);
    } else {
        event_kernel<R, false><<<need, SKG_EVENT_THREADS, 0, s>>>(W);
    }
#if SKG_LAUNCH_KERNEL
    {
        // a grid-stride pass: SKG_LAUNCH_OCC sizes it to the blocks that are resident at once
        static int sms = 0, per = 16;
        if (sms == 0) {
            int dev = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
#if SKG_LAUNCH_OCC
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, launch_kernel<R>, SKG_EVENT_THREADS, 0);
            if (per <= 0) per = 1;
#endif
        }
        launch_kernel<R><<<sms * per, SKG_EVENT_THREADS, 0, s>>>(W);
    }
#endif
    if (mid) cudaEventRecord(mid, s);
#if SKG_SPLIT_TRAV
    // the path jobs, then the peel-off jobs in their lean kernel
    trav_kernel<R, Stepper, 1, ONE><<<trav_blocks > 0 ? trav_blocks : resident_blocks<R, Stepper, 1, ONE>(smem), 256, smem, s>>>(W);
#if SKG_PDL
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(resident_blocks<R, Stepper, 2, ONE>(smem));
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaError_t e = cudaLaunchKernelEx(&cfg, trav_kernel<R, Stepper, 2, ONE>, W);
    if (e != cudaSuccess) return e;
#else
    trav_kernel<R, Stepper, 2, ONE><<<resident_blocks<R, Stepper, 2, ONE>(smem), 256, smem, s>>>(W);
#endif
#else
    trav_kernel<R, Stepper, 0, ONE><<<trav_blocks > 0 ? trav_blocks : resident_blocks<R, Stepper, 0, ONE>(smem), 256, smem, s>>>(W);
#endif
    return cudaGetLastError();
}

template<typename R, template<typename> class Stepper>
cudaError_t enqueue_tail(const WaveParams& W, cudaStream_t s) {
    tail_kernel<R, Stepper><<<(W.npool + 127) / 128, 128, 0, s>>>(W);
    return cudaGetLastError();
}

using WaveFn = cudaError_t (*)(const WaveParams&, int, int, cudaEvent_t, cudaStream_t);
using TailFn = cudaError_t (*)(const WaveParams&, cudaStream_t);
struct PassFns { WaveFn wave; TailFn tail; };

template<typename R, template<typename> class Stepper, bool ONE = false>
PassFns fns() { return {enqueue_wave<R, Stepper, ONE>, enqueue_tail<R, Stepper>}; }

// the FP32 tree and Voronoi walks have a single-slot instantiation (the grid as a kernel parameter:
// traversal pass of a phase, Voronoi disk 255 against 260 ms, k-d tree disk 1778 against 1800 ms,
// octree disk 1443 against 1445 ms; the Cartesian walk, 64.5 against 64.1 ms, keeps its shared copy)
template<template<typename> class Stepper>
PassFns fns32(bool one) { return one ? fns<float, Stepper, true>() : fns<float, Stepper, false>(); }

PassFns pick(int grid_type, int tree_walk, int precision, bool one) {
    const bool f64 = precision == SKG_PREC_FP64;
    switch (grid_type) {
    case SKG_GRID_CARTESIAN:
        if (f64) return fns<double, CartStepper>();
        return tree_walk == CW_UNIFORM ? fns<float, CartUniStepper>() : fns<float, CartStepper>();
    case SKG_GRID_OCTREE:
    case SKG_GRID_BINTREE:
        if (f64) return fns<double, TreeStepper>();
        if (tree_walk == TW_NODES) return fns<float, TreeNodeWalk>();
        if (tree_walk == TW_LATTICE) return fns32<TreeLatticeStepper>(one);
        return fns32<TreeStepper>(one);
    default:
        return f64 ? fns<double, VoronoiStepper>() : fns32<VoronoiStepper>(one);
    }
}

}  // namespace

WaveRunner::~WaveRunner() {
    for (cudaEvent_t e : ev_) cudaEventDestroy(e);
    for (cudaEvent_t e : tail_ev_) if (e) cudaEventDestroy(e);
    // (a runner that never reserved frees nothing: no device-wide synchronisation)
    for (void* p : {(void*)pk_, (void*)free_, (void*)ckpt_, (void*)ctr_}) if (p) cudaFree(p);
    for (int b = 0; b < 2; b++)
        for (void* p : {(void*)jobs_[b], (void*)jtau_[b], (void*)jL_[b]}) if (p) cudaFree(p);
    if (h_ctr_) cudaFreeHost(h_ctr_);
    if (copied_) cudaEventDestroy(copied_);
}

// grids whose FP32 walk resumes from checkpoints (the steppers' Resumable trait)
static bool ckpt_grid(int grid_type) {
    if (grid_type == SKG_GRID_VORONOI) return Resumable<VoronoiStepper<float>>::value;
    if (grid_type == SKG_GRID_CARTESIAN) return Resumable<CartStepper<float>>::value;
    return Resumable<TreeLatticeStepper<float>>::value;
}

cudaError_t WaveRunner::reserve(size_t pool, int ngroups, int grid_type) {
    cudaError_t e;
    if (!ctr_) {
        if ((e = cudaMalloc(&ctr_, NCTR * sizeof(unsigned))) != cudaSuccess) return e;
        if ((e = cudaMallocHost((void**)&h_ctr_, NCTR * sizeof(unsigned))) != cudaSuccess) return e;
        if ((e = cudaEventCreateWithFlags(&copied_, cudaEventDisableTiming)) != cudaSuccess) return e;
    }
    if (pool > cap_pool_) {
        cudaFree(pk_); pk_ = nullptr; cudaFree(free_); free_ = nullptr; cap_pool_ = 0;
        if ((e = cudaMalloc(&pk_, pool * sizeof(Packet))) != cudaSuccess) return e;
        if ((e = cudaMalloc(&free_, 2 * pool * sizeof(int))) != cudaSuccess) return e;
        cap_pool_ = pool;
    }
    if (SKG_CKPT && ckpt_grid(grid_type) && pool > cap_ckpt_) {
        cudaFree(ckpt_); ckpt_ = nullptr; cap_ckpt_ = 0;
        if ((e = cudaMalloc(&ckpt_, pool * SKG_CKPT_N * 2 * sizeof(float4))) != cudaSuccess) return e;
        cap_ckpt_ = pool;
    }
    const size_t jobs = pool * (size_t)(ngroups + 1);
    if (jobs > cap_jobs_) {
        for (int b = 0; b < 2; b++) {
            cudaFree(jobs_[b]); cudaFree(jtau_[b]); cudaFree(jL_[b]);
            jobs_[b] = nullptr; jtau_[b] = nullptr; jL_[b] = nullptr;
        }
        cap_jobs_ = 0;
        for (int b = 0; b < 2; b++) {
            if ((e = cudaMalloc(&jobs_[b], jobs * sizeof(int2))) != cudaSuccess) return e;
            if ((e = cudaMalloc(&jtau_[b], jobs * sizeof(double))) != cudaSuccess) return e;
            if ((e = cudaMalloc(&jL_[b], jobs * sizeof(double))) != cudaSuccess) return e;
        }
        cap_jobs_ = jobs;
    }
    return cudaSuccess;
}

cudaError_t WaveRunner::enqueue(int n) {
    WaveFn fn = pick(grid_type_, tree_walk_, precision_, one_).wave;
    cudaError_t e;
    for (int i = 0; i < n; i++) {
        const int w = waves_ + i, b = w & 1;
        WaveParams W;
        W.R = P_; W.pk = pk_; W.npool = npool_; W.wave = w;
        W.jobs = jobs_[b]; W.jtau = jtau_[b]; W.jL = jL_[b]; W.jcount = ctr_ + 8 * b;
        W.pjobs = jobs_[b ^ 1]; W.pjtau = jtau_[b ^ 1]; W.pjL = jL_[b ^ 1];
        W.last_busy = ctr_ + 16;
        W.freelist = free_; W.intlist = free_ + npool_; W.ckpt = ckpt_on_ ? ckpt_ : nullptr;
        W.g0 = g0_;
        if ((e = cudaMemsetAsync(ctr_ + 8 * b, 0, 8 * sizeof(unsigned), stream_)) != cudaSuccess) return e;
        if (timed_) {
            while (ev_.size() < 3 * (size_t)(w + 1)) {
                cudaEvent_t x;
                if ((e = cudaEventCreate(&x)) != cudaSuccess) return e;
                ev_.push_back(x);
            }
            if ((e = cudaEventRecord(ev_[3 * w], stream_)) != cudaSuccess) return e;
        }
        if ((e = fn(W, nslots_, trav_blocks_, timed_ ? ev_[3 * w + 1] : nullptr, stream_)) != cudaSuccess) return e;
        if (timed_ && (e = cudaEventRecord(ev_[3 * w + 2], stream_)) != cudaSuccess) return e;
    }
    waves_ += n;
    if ((e = cudaMemcpyAsync(h_ctr_, ctr_, NCTR * sizeof(unsigned), cudaMemcpyDeviceToHost, stream_)) != cudaSuccess) return e;
    // inside stream capture the record must become a graph node that the host can wait on
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if ((e = cudaStreamIsCapturing(stream_, &cs)) != cudaSuccess) return e;
    return cs == cudaStreamCaptureStatusNone ? cudaEventRecord(copied_, stream_)
                                             : cudaEventRecordWithFlags(copied_, stream_, cudaEventRecordExternal);
}

cudaError_t WaveRunner::begin(const RunParams& P, int grid_type, int tree_walk, int precision, int nslots,
                              size_t npool, int trav_blocks, cudaStream_t s, const DevGrid* one_grid) {
    if (npool == 0 || npool > cap_pool_) return cudaErrorInvalidValue;
    P_ = P; grid_type_ = grid_type; tree_walk_ = tree_walk; precision_ = precision; nslots_ = nslots;
    one_ = one_grid != nullptr && nslots == 1;
    if (one_) g0_ = *one_grid; else std::memset(&g0_, 0, sizeof(g0_));
    trav_blocks_ = trav_blocks; stream_ = s; npool_ = (int)npool; waves_ = 0; tail_ran_ = false;
    const char* td = std::getenv("SKG_TAIL_DIV");
    tail_div_ = td ? std::atoi(td) : tail_div;
    const char* ck = std::getenv("SKG_CKPT");
    ckpt_on_ = !(ck && std::atoi(ck) == 0) && ckpt_ && cap_ckpt_ >= (size_t)npool;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(s, &cs);
    timed_ = timing && cs == cudaStreamCaptureStatusNone;
    cudaError_t e;
    if ((e = cudaMemsetAsync(pk_, 0, npool * sizeof(Packet), s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(ctr_, 0, NCTR * sizeof(unsigned), s)) != cudaSuccess) return e;
    pending_ = true;
    return enqueue(estimate);
}

cudaError_t WaveRunner::enqueue_tail() {
    const int b = (waves_ - 1) & 1;               // the last wave's jobs hold the pending peel-offs
    WaveParams W;
    W.R = P_; W.pk = pk_; W.npool = npool_; W.wave = waves_;
    W.jobs = nullptr; W.jtau = nullptr; W.jL = nullptr; W.jcount = ctr_ + 8 * (b ^ 1);
    W.pjobs = jobs_[b]; W.pjtau = jtau_[b]; W.pjL = jL_[b];
    W.last_busy = ctr_ + 16;
    W.freelist = nullptr; W.intlist = nullptr; W.ckpt = ckpt_on_ ? ckpt_ : nullptr;
    cudaError_t e;
    if (timed_) {
        for (int i = 0; i < 2; i++)
            if (!tail_ev_[i] && (e = cudaEventCreate(&tail_ev_[i])) != cudaSuccess) return e;
        if ((e = cudaEventRecord(tail_ev_[0], stream_)) != cudaSuccess) return e;
    }
    W.g0 = g0_;
    if ((e = pick(grid_type_, tree_walk_, precision_, one_).tail(W, stream_)) != cudaSuccess) return e;
    tail_ran_ = true;
    return timed_ ? cudaEventRecord(tail_ev_[1], stream_) : cudaSuccess;
}

cudaError_t WaveRunner::finish(int timeout_ms, cudaEvent_t end, bool* timed_out) {
    if (timed_out) *timed_out = false;
    const auto t0 = std::chrono::steady_clock::now();
    bool more = false;                            // waves were added after the caller's end event
    while (pending_) {
        while (true) {
            const cudaError_t q = cudaEventQuery(copied_);
            if (q == cudaSuccess) break;
            if (q != cudaErrorNotReady) return q;
            if (timeout_ms >= 0 &&
                std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count() > timeout_ms) {
                if (timed_out) *timed_out = true;
                return cudaSuccess;
            }
            std::this_thread::sleep_for(std::chrono::microseconds(50));
        }
        const unsigned busy = h_ctr_[8 * ((waves_ - 1) & 1) + 3];
        if (busy == 0) {
            pending_ = false;
            estimate = (int)h_ctr_[16] + 3;        // the last busy wave, the detection wave, one spare
            break;
        }
        if (tail_div_ > 0 && (size_t)busy * (size_t)tail_div_ <= (size_t)npool_) {
            // few packets left in flight: the tail pass finishes them (and any packets still to
            // launch) in one launch; the next phase enqueues this many waves before it looks
            cudaError_t e = enqueue_tail();
            pending_ = false;
            if (e != cudaSuccess) return e;
            estimate = waves_;
            more = true;
            break;
        }
        cudaError_t e = enqueue(estimate > 32 ? estimate / 4 : 8);
        if (e != cudaSuccess) { pending_ = false; return e; }
        more = true;
    }
    return (end && more) ? cudaEventRecord(end, stream_) : cudaSuccess;
}

cudaError_t WaveRunner::times(float* event_ms, float* trav_ms) const {
    float a = 0, t = 0;
    if (timed_ && !pending_) {
        for (int w = 0; w < waves_; w++) {
            float x = 0, y = 0;
            cudaError_t e = cudaEventElapsedTime(&x, ev_[3 * w], ev_[3 * w + 1]);
            if (e == cudaSuccess) e = cudaEventElapsedTime(&y, ev_[3 * w + 1], ev_[3 * w + 2]);
            if (e != cudaSuccess) return e;
            a += x; t += y;
        }
        if (tail_ran_) {
            float y = 0;
            cudaError_t e = cudaEventElapsedTime(&y, tail_ev_[0], tail_ev_[1]);
            if (e != cudaSuccess) return e;
            t += y;
        }
    }
    if (event_ms) *event_ms = a;
    if (trav_ms) *trav_ms = t;
    return cudaSuccess;
}

}  // namespace skg
