// skg_tracer.cu -- the persistent photon-packet tracer.
//
// One launch runs a whole phase (stellar emission, dust self-absorption or dust emission) for a
// batch of wavelengths of one or more simulations: it replaces
// Parallel::call(this, &dostellaremissionchunk, Nlambda, Nchunks) (MonteCarloSimulation.cpp:241-295)
// and the two dust chunk bodies (PanMonteCarloSimulation.cpp:191-346).  Each thread carries one
// packet at a time through an explicit state machine:
//
//   FETCH -> launch -> PEEL(emission) x groups -> MAIN1 -> [terminate?] -> MAIN2 -> PEEL(scattering)
//         -> SCATTER -> MAIN1 -> ...
//
// and every lane of a warp executes the same cell-step code whatever traversal it is on (a
// peel-off ray, the full path of the packet, or the re-walk to the interaction point), so the
// inner loop stays converged.  Cell steps never materialise the segment list:
//   MAIN1 streams kappa*rho*ds into the FP64 cumulative optical depth and the per-cell absorption
//         tallies (MonteCarloSimulation::simulateescapeandabsorption, :432-509);
//   MAIN2 re-walks the same path until the cumulative optical depth passes the sampled one and
//         interpolates inside that segment -- DustGridPath::pathlength (DustGridPath.cpp:162-173);
//   PEEL  accumulates the optical depth towards an observer (DustSystem::opticaldepth, :960-976).
// Instruments seen from the same direction share one peel-off traversal (identical optical
// depth; the reference recomputes it per instrument).  The event code (launch samplers,
// scattering, detection) sits in non-inlined functions so that the step loop keeps few registers.
#include "skg_scene.cuh"
#include "skg_internal.h"

namespace skg {

#ifndef SKG_EVENT_LANES
#define SKG_EVENT_LANES 32
#endif
#ifndef SKG_TRACER_MIN_BLOCKS
#define SKG_TRACER_MIN_BLOCKS 3
#endif

enum Mode : int { M_FETCH = 0, M_LAUNCH, M_PEEL_NEXT, M_MAIN1_START, M_AFTER_MAIN1, M_AFTER_MAIN2, M_SCATTER, M_DONE };
enum Trav : int { T_NONE = 0, T_PEEL, T_MAIN1, T_MAIN2 };
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

// Instrument::detect for the members of one direction group after the shared traversal
// (SEDInstrument.cpp:32-42, FrameInstrument.cpp:33-47, SimpleInstrument.cpp:35-49,
// FullInstrument.cpp:109-177).  Returns the number of tally updates.
__device__ __noinline__ int detect_group(const DevScene& S, int grp, int ell, double Lpeel, double tau,
                                         int nscatt_peel, bool stellar, double x, double y, double z) {
    double Lextf = Lpeel * exp(-tau);
    const int nl = S.nlambda;
    int adds = 0;
    for (int q = S.group_start[grp]; q < S.group_start[grp + 1]; q++) {
        const DevInstr& I = S.instr[S.group_instr[q]];
        int l = (I.type == SKG_INSTR_SED) ? -1 : pixel_on_detector(I, x, y, z);
        size_t fp = (size_t)I.nxp * I.nyp;
        if (I.type == SKG_INSTR_FRAME) {
            if (l >= 0) { atomicAdd(I.cube + (size_t)ell * fp + l, Lextf); adds++; }
        } else if (I.type == SKG_INSTR_SED) {
            atomicAdd(I.sed + ell, Lextf); adds++;
        } else if (I.type == SKG_INSTR_SIMPLE) {
            atomicAdd(I.sed + ell, Lextf); adds++;
            if (l >= 0) { atomicAdd(I.cube + (size_t)ell * fp + l, Lextf); adds++; }
        } else {
            auto add = [&](int c, double v) {
                atomicAdd(I.sed + (size_t)c * nl + ell, v); adds++;
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

// Does the group need a traversal?  Frame-only groups skip it when the packet projects off every
// frame (FrameInstrument.cpp:36-37).
SKG_D bool group_needs_traversal(const DevScene& S, int grp, double x, double y, double z) {
    if (!S.group_frame_only[grp]) return true;
    for (int q = S.group_start[grp]; q < S.group_start[grp + 1]; q++)
        if (pixel_on_detector(S.instr[S.group_instr[q]], x, y, z) >= 0) return true;
    return false;
}

struct Launched { double x, y, z, kx, ky, kz, L, Lth; int ok; int stellar; };

// Packet launch: StellarSystem::launch (StellarSystem.cpp:116-158) with the geometry samplers
// (GeometricStellarComp.cpp:75-81), or a dust-emission launch from the cell luminosity CDF
// (PanMonteCarloSimulation.cpp:216-224 self-absorption, :301-323 emission with bias).
__device__ __noinline__ Launched launch_packet(const DevGrid& g, const DevScene& S, int phase, int ell,
                                               uint64_t Npp_total, Philox& rng) {
    Launched o;
    o.ok = 0;
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
        o.L = Lw; o.stellar = 1;
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
__device__ __noinline__ double sample_interaction(double xi, double taupath, double& L, Philox& rng) {
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

template<typename R, template<typename> class Stepper>
__global__ void __launch_bounds__(256, SKG_TRACER_MIN_BLOCKS)
tracer_kernel(const RunParams P) {
    extern __shared__ unsigned char smem_raw[];
    DevGrid* sg = reinterpret_cast<DevGrid*>(smem_raw);
    __shared__ const DevScene* s_scene[MAX_SLOTS];
    __shared__ unsigned long long s_cnt[C_N];
    const BatchHeader H = *P.hdr;
    for (int i = threadIdx.x; i < C_N; i += blockDim.x) s_cnt[i] = 0;
    for (int i = threadIdx.x; i < H.nslots; i += blockDim.x) { sg[i] = P.grids[i]; s_scene[i] = P.scenes[i]; }
    __syncthreads();

    const int lane = threadIdx.x & 31;
    const int phase = H.phase;
    const bool peel_on = phase != SKG_PHASE_DUST_SELFABS;

    Philox rng;
    int slot = 0;
    double L = 0, Lth = 0, Lpeel = 0, Lsca_acc = 0;
    int ell = 0, nscatt = 0, grp = 0;
    bool stellar = true, scat_peel = false;
    V3<R> r = mk3((R)0, (R)0, (R)0), k = mk3((R)0, (R)0, (R)1);
    int mode = M_FETCH, trav = T_NONE;
    int int_cell = -1;
    int pos_cell = -2;          // cell holding the packet position: -2 unknown, -1 outside the grid
    uint64_t Npp_total = 1;
    double tau = 0, s = 0, tau_int = 0, s_int = 0;
    Stepper<R> st;
    unsigned c_steps = 0;

    while (true) {
        // ---------------- event processing: runs until a traversal starts or no work is left.
        // A lane whose traversal ended waits (idle in the step below) until SKG_EVENT_LANES lanes
        // of the warp, or all of its live lanes, are waiting, so that the divergent event code is
        // paid once for many lanes instead of once per finished traversal.
        const unsigned live = __activemask();
        const unsigned waiting = __ballot_sync(live, trav == T_NONE);
        const bool run_events = __popc(waiting) >= SKG_EVENT_LANES || waiting == live;
        while (run_events && trav == T_NONE && mode != M_DONE) {
            const DevGrid& g = sg[slot];
            const DevScene& S = *s_scene[slot];
            switch (mode) {
            case M_FETCH: {
                unsigned mask = __activemask();
                int leader = __ffs(mask) - 1;
                unsigned long long base = 0;
                if (lane == leader) base = atomicAdd(P.work, (unsigned long long)__popc(mask));
                base = __shfl_sync(mask, base, leader);
                uint64_t p = base + __popc(mask & ((1u << lane) - 1));
                if (p >= H.total) { mode = M_DONE; break; }
                int it = find_item(P.items, H.nitems, p);
                const WorkItem W = P.items[it];
                uint64_t q = p - W.begin;
                int ei = (int)(q / W.count);
                uint64_t ip = W.first + (q - (uint64_t)ei * W.count);
                slot = W.slot;
                ell = P.ells[W.ell0 + ei];
                Npp_total = W.npp_total;
                rng.init(W.seed, ip, (uint32_t)ell | ((uint32_t)phase << 24));
                atomicAdd(&s_cnt[C_PACKETS], 1ull);
                mode = M_LAUNCH;        // the launch runs with the packet's own slot bound
                break;
            }
            case M_LAUNCH: {
                Launched o = launch_packet(g, S, phase, ell, Npp_total, rng);
                if (!o.ok) { mode = M_FETCH; break; }
                L = o.L; Lth = o.Lth; stellar = o.stellar;
                r = mk3((R)o.x, (R)o.y, (R)o.z);
                k = mk3((R)o.kx, (R)o.ky, (R)o.kz);
                nscatt = 0; pos_cell = -2; int_cell = -1;
                if (peel_on) { mode = M_PEEL_NEXT; grp = 0; scat_peel = false; }
                else mode = M_MAIN1_START;
                break;
            }
            case M_PEEL_NEXT: {
                // one traversal per direction group (MonteCarloSimulation.cpp:299-357)
                while (grp < S.ngroups) {
                    double w = 1.0;
                    if (scat_peel) {
                        w = peel_weight(S, ell, int_cell, (double)k.x, (double)k.y, (double)k.z, S.gkx[grp], S.gky[grp],
                                        S.gkz[grp]);
                        if (w < 0) { grp = S.ngroups; break; }   // abort peel-off
                    }
                    Lpeel = L * w;
                    if (group_needs_traversal(S, grp, (double)r.x, (double)r.y, (double)r.z)) {
                        st.init(g, r.x, r.y, r.z, (R)S.gkx[grp], (R)S.gky[grp], (R)S.gkz[grp], pos_cell);
                        if (pos_cell == -2) pos_cell = st.cell0;
                        trav = T_PEEL; tau = 0;
                        break;
                    }
                    grp++;
                }
                if (trav == T_NONE) mode = scat_peel ? M_SCATTER : M_MAIN1_START;
                break;
            }
            case M_MAIN1_START: {
                if (S.ncomp == 0) { mode = M_FETCH; break; }
                st.init(g, r.x, r.y, r.z, k.x, k.y, k.z, pos_cell);
                if (pos_cell == -2) pos_cell = st.cell0;
                trav = T_MAIN1; tau = 0; Lsca_acc = 0;
                break;
            }
            case M_AFTER_MAIN1: {
                double taupath = tau;
                if (taupath < 0.0 || isnan(taupath) || isinf(taupath)) {   // DustSystem.cpp:953-955
                    atomicOr(P.err, ERR_NAN_TAU); atomicAdd(&s_cnt[C_ERR], 1ull); mode = M_FETCH; break;
                }
                if (S.ncomp == 1) L = L * S.albedo[ell] * (-expm1(-taupath));   // :441-462
                else L = Lsca_acc;
                if (L <= 0 || (L <= Lth && nscatt >= S.min_scatt_events)) { mode = M_FETCH; break; }
                if (nscatt >= P.max_scatt) {
                    atomicOr(P.err, ERR_SCATT_BUDGET); atomicAdd(&s_cnt[C_ERR], 1ull); mode = M_FETCH; break;
                }
                if (taupath == 0.0) { s_int = 0; mode = M_AFTER_MAIN2; break; }
                tau_int = sample_interaction(S.xi, taupath, L, rng);
                st.init(g, r.x, r.y, r.z, k.x, k.y, k.z, pos_cell);
                trav = T_MAIN2; tau = 0; s = 0; s_int = -1; int_cell = -1;
                break;
            }
            case M_AFTER_MAIN2: {
                R si = (R)s_int;
                r = mk3(r.x + si * k.x, r.y + si * k.y, r.z + si * k.z);   // PhotonPackage::propagate
                // the interaction point lies in the cell of its segment (verified by the stepper)
                if (s_int > 0) pos_cell = (int_cell >= 0) ? int_cell : -2;
                if (peel_on) { mode = M_PEEL_NEXT; grp = 0; scat_peel = true; }
                else mode = M_SCATTER;
                break;
            }
            case M_SCATTER: {
                V3<double> kn = scatter_direction(S, ell, int_cell, mk3((double)k.x, (double)k.y, (double)k.z), rng);
                k = mk3((R)kn.x, (R)kn.y, (R)kn.z);
                nscatt++;
                atomicAdd(&s_cnt[C_SCATT], 1ull);
                mode = M_MAIN1_START;
                break;
            }
            default: break;
            }
        }
        if (mode == M_DONE) break;
        if (trav == T_NONE) continue;

        // ---------------- one cell step of the current traversal
        const DevGrid& g = sg[slot];
        const DevScene& S = *s_scene[slot];
        int m; R ds;
        if (st.next(g, m, ds)) {
            c_steps++;
            // one dust component: the FP32 tree walk carries the cell density in its leaf record
            double kr = (S.ncomp == 1 && st.rho >= 0.f) ? S.kext[ell] * (double)st.rho : kappa_rho<R>(S, m, ell);
            double dtau = kr * (double)ds;
            if (trav == T_PEEL) {
                tau += dtau;
            } else if (trav == T_MAIN1) {
                if (m >= 0) {
                    const bool store = (phase == SKG_PHASE_STELLAR) ? (S.store_abs != 0) : (phase == SKG_PHASE_DUST_SELFABS);
                    if (S.ncomp == 1) {
                        if (store) {
                            double Lintm = L * exp(-tau) * (-expm1(-dtau));
                            double* labs = (phase == SKG_PHASE_STELLAR) ? S.labs_stel : S.labs_dust;
                            atomicAdd(labs + (size_t)m * S.nlambda + ell, (1.0 - S.albedo[ell]) * Lintm);
                            atomicAdd(&s_cnt[C_ABS], 1ull);
                        }
                    } else {
                        double ksca = 0, kext = 0;
                        for (int h = 0; h < S.ncomp; h++) {
                            double rh = rho_load<R>(S, (size_t)h * S.ncells + m);
                            ksca += rh * S.ksca[h * S.nlambda + ell]; kext += rh * S.kext[h * S.nlambda + ell];
                        }
                        double alb = (kext > 0.0) ? ksca / kext : 0.0;
                        double Lintm = L * exp(-tau) * (-expm1(-dtau));
                        Lsca_acc += alb * Lintm;
                        if (store) {
                            double* labs = (phase == SKG_PHASE_STELLAR) ? S.labs_stel : S.labs_dust;
                            atomicAdd(labs + (size_t)m * S.nlambda + ell, (1.0 - alb) * Lintm);
                            atomicAdd(&s_cnt[C_ABS], 1ull);
                        }
                    }
                }
                tau += dtau;
            } else {  // T_MAIN2
                double tn = tau + dtau, sn = s + (double)ds;
                if (tn > tau_int) {
                    s_int = s + ((tau_int - tau) / (tn - tau)) * (sn - s);
                    int_cell = m;
                    trav = T_NONE; mode = M_AFTER_MAIN2;
                    atomicAdd(&s_cnt[C_TRAV], 1ull);
                    atomicAdd(&s_cnt[C_NBR], (unsigned long long)st.scanned);
                    atomicAdd(&s_cnt[C_FB], (unsigned long long)st.fallbacks);
                } else { tau = tn; s = sn; }
            }
        } else {
            // traversal ended
            atomicAdd(&s_cnt[C_TRAV], 1ull);
            atomicAdd(&s_cnt[C_NBR], (unsigned long long)st.scanned);
            atomicAdd(&s_cnt[C_FB], (unsigned long long)st.fallbacks);
            if (st.steps > g.max_steps) { atomicOr(P.err, ERR_STEP_BUDGET); atomicAdd(&s_cnt[C_ERR], 1ull); }
            if (trav == T_PEEL) {
                int adds = detect_group(S, grp, ell, Lpeel, tau, scat_peel ? nscatt + 1 : 0, stellar,
                                        (double)r.x, (double)r.y, (double)r.z);
                atomicAdd(&s_cnt[C_PIX], (unsigned long long)adds);
                atomicAdd(&s_cnt[C_PEEL], 1ull);
                grp++;
                mode = M_PEEL_NEXT;
            } else if (trav == T_MAIN1) {
                mode = M_AFTER_MAIN1;
            } else {
                s_int = s;  // DustGridPath::pathlength: tau beyond the last segment -> full length
                mode = M_AFTER_MAIN2;
            }
            trav = T_NONE;
        }
    }

    atomicAdd(&s_cnt[C_STEPS], (unsigned long long)c_steps);
    __syncthreads();
    if (threadIdx.x < C_N) atomicAdd(P.counters + threadIdx.x, s_cnt[threadIdx.x]);
}

// ---------------------------------------------------------------------------------------------
template<typename R, template<typename> class Stepper>
static cudaError_t launch_one(const RunParams& P, int nslots, int blocks, int threads, cudaStream_t stream) {
    auto kern = tracer_kernel<R, Stepper>;
    size_t smem = (size_t)nslots * sizeof(DevGrid);
    if (blocks <= 0) {
        int dev = 0, sms = 0, per = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, threads, smem);
        blocks = sms * (per > 0 ? per : 1);
    }
    kern<<<blocks, threads, smem, stream>>>(P);
    return cudaGetLastError();
}

cudaError_t launch_tracer(int grid_type, bool bookkeeping, const RunParams& P, int nslots, int precision, int blocks,
                          int threads, cudaStream_t stream) {
    if (threads <= 0) threads = 256;
    bool f64 = precision == SKG_PREC_FP64;
    switch (grid_type) {
    case SKG_GRID_CARTESIAN:
        return f64 ? launch_one<double, CartStepper>(P, nslots, blocks, threads, stream)
                   : launch_one<float, CartStepper>(P, nslots, blocks, threads, stream);
    case SKG_GRID_OCTREE:
    case SKG_GRID_BINTREE:
        if (f64) return launch_one<double, TreeStepper>(P, nslots, blocks, threads, stream);
        return bookkeeping ? launch_one<float, TreeNodeWalk>(P, nslots, blocks, threads, stream)
                           : launch_one<float, TreeStepper>(P, nslots, blocks, threads, stream);
    default:
        return f64 ? launch_one<double, VoronoiStepper>(P, nslots, blocks, threads, stream)
                   : launch_one<float, VoronoiStepper>(P, nslots, blocks, threads, stream);
    }
}

}  // namespace skg
