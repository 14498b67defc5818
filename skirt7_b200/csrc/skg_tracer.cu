// skg_tracer.cu -- the persistent photon-packet tracer.
//
// One launch runs a whole phase (stellar emission, dust self-absorption or dust emission) for a
// batch of wavelengths: it replaces Parallel::call(this, &dostellaremissionchunk, Nlambda, Nchunks)
// (MonteCarloSimulation.cpp:241-295) and the two dust chunk bodies (PanMonteCarloSimulation.cpp:
// 191-346).  Each thread carries one packet at a time through an explicit state machine:
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
// depth; the reference recomputes it per instrument).
#include "skg_scene.cuh"
#include "skg_internal.h"

namespace skg {

enum Mode : int { M_FETCH = 0, M_PEEL_NEXT, M_MAIN1_START, M_AFTER_MAIN1, M_AFTER_MAIN2, M_SCATTER, M_DONE };
enum Trav : int { T_NONE = 0, T_PEEL, T_MAIN1, T_MAIN2 };

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

// Instrument::detect for the members of one direction group after the shared traversal.
SKG_D void detect_group(const DevScene& S, int grp, int ell, double Lpeel, double tau, int nscatt_peel,
                        bool stellar, double x, double y, double z, unsigned& c_pix) {
    double extf = exp(-tau);
    double Lextf = Lpeel * extf;
    const int nl = S.nlambda;
    for (int q = S.group_start[grp]; q < S.group_start[grp + 1]; q++) {
        const DevInstr& I = S.instr[S.group_instr[q]];
        int l = (I.type == SKG_INSTR_SED) ? -1 : pixel_on_detector(I, x, y, z);
        size_t fp = (size_t)I.nxp * I.nyp;
        if (I.type == SKG_INSTR_FRAME) {                       // FrameInstrument.cpp:33-47
            if (l >= 0) { atomicAdd(I.cube + (size_t)ell * fp + l, Lextf); c_pix++; }
        } else if (I.type == SKG_INSTR_SED) {                  // SEDInstrument.cpp:32-42
            atomicAdd(I.sed + ell, Lextf); c_pix++;
        } else if (I.type == SKG_INSTR_SIMPLE) {               // SimpleInstrument.cpp:35-49
            atomicAdd(I.sed + ell, Lextf); c_pix++;
            if (l >= 0) { atomicAdd(I.cube + (size_t)ell * fp + l, Lextf); c_pix++; }
        } else {                                               // FullInstrument.cpp:109-177
            auto add = [&](int c, double v) {
                atomicAdd(I.sed + (size_t)c * nl + ell, v); c_pix++;
                if (l >= 0) { atomicAdd(I.cube + ((size_t)c * nl + ell) * fp + l, v); c_pix++; }
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
}

// Does the group need a traversal?  Frame-only groups skip it when the packet projects off every
// frame (FrameInstrument.cpp:36-37).
SKG_D bool group_needs_traversal(const DevScene& S, int grp, double x, double y, double z) {
    if (!S.group_frame_only[grp]) return true;
    for (int q = S.group_start[grp]; q < S.group_start[grp + 1]; q++)
        if (pixel_on_detector(S.instr[S.group_instr[q]], x, y, z) >= 0) return true;
    return false;
}

template<typename R, template<typename> class Stepper>
__global__ void __launch_bounds__(256)
tracer_kernel(const DevGrid g, const DevScene* __restrict__ Sp, const RunParams P) {
    const DevScene& S = *Sp;
    __shared__ unsigned long long s_cnt[10];
    if (threadIdx.x < 10) s_cnt[threadIdx.x] = 0;
    __syncthreads();

    const int lane = threadIdx.x & 31;
    const uint64_t total = (uint64_t)P.nell * P.npp;
    const int nl = S.nlambda;
    const bool dust_phase = P.phase != SKG_PHASE_STELLAR;
    const bool store = (P.phase == SKG_PHASE_STELLAR) ? (S.store_abs != 0) : (P.phase == SKG_PHASE_DUST_SELFABS);
    double* labs = (P.phase == SKG_PHASE_STELLAR) ? S.labs_stel : S.labs_dust;
    const bool peel_on = P.phase != SKG_PHASE_DUST_SELFABS;

    Philox rng;
    double L = 0, Lth = 0, Lpeel = 0, Lsca_acc = 0;
    int ell = 0, nscatt = 0, grp = 0;
    bool stellar = true, scat_peel = false;
    V3<R> r = mk3((R)0, (R)0, (R)0), k = mk3((R)0, (R)0, (R)1);
    int mode = M_FETCH, trav = T_NONE;
    int int_cell = -1;
    int pos_cell = -2;          // cell holding the packet position: -2 unknown, -1 outside the grid
    double tau = 0, s = 0, tau_int = 0, s_int = 0;
    Stepper<R> st;
    unsigned c_steps = 0, c_trav = 0, c_scatt = 0, c_peel = 0, c_abs = 0, c_pix = 0, c_nbr = 0, c_fb = 0,
             c_err = 0, c_pk = 0;

    while (true) {
        // ---------------- event processing: runs until a traversal starts or no work is left
        while (trav == T_NONE && mode != M_DONE) {
            switch (mode) {
            case M_FETCH: {
                unsigned mask = __activemask();
                int leader = __ffs(mask) - 1;
                unsigned long long base = 0;
                if (lane == leader) base = atomicAdd(P.work, (unsigned long long)__popc(mask));
                base = __shfl_sync(mask, base, leader);
                uint64_t p = base + __popc(mask & ((1u << lane) - 1));
                if (p >= total) { mode = M_DONE; break; }
                int ei = (int)(p / P.npp);
                uint64_t ip = p - (uint64_t)ei * P.npp;
                ell = P.ells[ei];
                rng.init(P.seed, P.first_packet + ip, (uint32_t)ell | ((uint32_t)P.phase << 24));
                c_pk++;
                pos_cell = -2;
                nscatt = 0;
                V3<double> pos, dir;
                if (!dust_phase) {
                    // StellarSystem::launch (StellarSystem.cpp:116-158)
                    double Lpp = S.Lv[ell] / (double)P.Npp_total;
                    if (!(Lpp > 0)) break;                       // mode stays FETCH
                    Lth = Lpp / S.min_weight_reduction;
                    int N = S.nstellar, h = 0;
                    double Lw = Lpp;
                    if (N > 1) {
                        double eb = S.emission_bias;
                        double X = rng.uniform();
                        if (X < eb) h = max(0, min(N - 1, (int)(N * X / eb)));
                        else h = dlocate_clip(S.Xvv + (size_t)ell * (N + 1), N + 1, (X - eb) / (1.0 - eb));
                        double Lh = S.starL[h * nl + ell];
                        if (!(Lh > 0)) break;                    // launched with zero luminosity
                        Lw = Lpp * (1.0 / (1.0 - eb + eb * (S.Lv[ell] / N) / Lh));
                    }
                    pos = geom_position(S.stellar[h], rng);      // GeometricStellarComp.cpp:75-81
                    dir = iso_direction(rng);
                    L = Lw; stellar = true;
                } else {
                    // PanMonteCarloSimulation.cpp:216-224 (self-absorption), :301-323 (emission)
                    double Ltot = S.emit_Ltot[ell];
                    if (!(Ltot > 0)) break;
                    double Lem = Ltot / (double)P.Npp_total;
                    Lth = Lem / S.min_weight_reduction;
                    const int nc = S.ncells;
                    const double* cdf = S.emit_cdf + (size_t)ell * (nc + 1);
                    double X = rng.uniform(), weight = 1.0;
                    int m;
                    if (P.phase == SKG_PHASE_DUST_SELFABS) m = dlocate_clip(cdf, nc + 1, X);
                    else {
                        double xi = S.dust_emission_bias;
                        if (X < xi) m = max(0, min(nc - 1, (int)(nc * X / xi)));
                        else m = dlocate_clip(cdf, nc + 1, (X - xi) / (1 - xi));
                        double Lmean = Ltot / nc;
                        weight = 1.0 / (1 - xi + xi * Lmean / S.emit_Lv[(size_t)ell * nc + m]);
                    }
                    L = Lem * weight;
                    if (!(L > 0)) break;
                    pos = random_position_in_cell(g, m, rng);
                    dir = iso_direction(rng);
                    stellar = false;
                }
                r = mk3((R)pos.x, (R)pos.y, (R)pos.z);
                k = mk3((R)dir.x, (R)dir.y, (R)dir.z);
                if (peel_on) { mode = M_PEEL_NEXT; grp = 0; scat_peel = false; }
                else mode = M_MAIN1_START;
                break;
            }
            case M_PEEL_NEXT: {
                // one traversal per direction group (MonteCarloSimulation.cpp:299-357)
                while (grp < S.ngroups) {
                    double w = 1.0;
                    if (scat_peel) {
                        double gx_ = S.gkx[grp], gy_ = S.gky[grp], gz_ = S.gkz[grp];
                        double cosalpha = (double)k.x * gx_ + (double)k.y * gy_ + (double)k.z * gz_;
                        if (S.ncomp == 1) {                       // DustMix.cpp:648-654
                            double gg = S.asym[ell];
                            double t = 1.0 + gg * gg - 2 * gg * cosalpha;
                            w = (1.0 - gg) * (1.0 + gg) / sqrt(t * t * t);
                        } else {                                  // weights kappa_sca*rho (:319-331)
                            double sum = 0, acc = 0;
                            for (int h = 0; h < S.ncomp; h++) {
                                double wv = (int_cell >= 0) ? S.ksca[h * nl + ell] * S.rho[(size_t)h * S.ncells + int_cell] : 0.0;
                                double gg = S.asym[h * nl + ell];
                                double t = 1.0 + gg * gg - 2 * gg * cosalpha;
                                acc += wv * (1.0 - gg) * (1.0 + gg) / sqrt(t * t * t);
                                sum += wv;
                            }
                            if (!(sum > 0)) { grp = S.ngroups; break; }   // abort peel-off
                            w = acc / sum;
                        }
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
                    atomicOr(P.err, ERR_NAN_TAU); c_err++; mode = M_FETCH; break;
                }
                if (S.ncomp == 1) L = L * S.albedo[ell] * (-expm1(-taupath));   // :441-462
                else L = Lsca_acc;
                if (L <= 0 || (L <= Lth && nscatt >= S.min_scatt_events)) { mode = M_FETCH; break; }
                if (nscatt >= P.max_scatt) { atomicOr(P.err, ERR_SCATT_BUDGET); c_err++; mode = M_FETCH; break; }
                if (taupath == 0.0) { s_int = 0; int_cell = -1; mode = M_AFTER_MAIN2; break; }
                // MonteCarloSimulation::simulatepropagation (:513-531), Random::exponcutoff (Random.cpp:163-176)
                double xi = S.xi, ti;
                auto expcut = [&](double xmax) -> double {
                    if (xmax < 1e-10) return rng.uniform() * xmax;
                    double x;
                    int guard = 0;
                    do { x = -log1p(-rng.uniform() * (-expm1(-xmax))); } while (x > xmax && ++guard < 64);
                    return fmin(x, xmax);
                };
                if (xi == 0.0) ti = expcut(taupath);
                else {
                    double X = rng.uniform();
                    ti = (X < xi) ? rng.uniform() * taupath : expcut(taupath);
                    double p = -exp(-ti) / expm1(-taupath);
                    double q = (1.0 - xi) * p + xi / taupath;
                    L *= p / q;
                }
                tau_int = ti;
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
                // DustSystem::randomMixForPosition (DustSystem.cpp:855-869) + HG (DustMix.cpp:595-602)
                int h = 0;
                if (S.ncomp > 1 && int_cell >= 0) {
                    double tot = 0, pv[MAX_COMP];
                    for (int c = 0; c < S.ncomp; c++) { pv[c] = S.ksca[c * nl + ell] * S.rho[(size_t)c * S.ncells + int_cell]; tot += pv[c]; }
                    double X = rng.uniform(), acc = 0;
                    for (h = 0; h < S.ncomp - 1; h++) { acc += pv[h] / tot; if (X < acc) break; }
                }
                double gg = S.asym[h * nl + ell];
                V3<double> kd = mk3((double)k.x, (double)k.y, (double)k.z), kn;
                if (fabs(gg) < 1e-6) kn = iso_direction(rng);
                else {
                    double f = ((1.0 - gg) * (1.0 + gg)) / (1.0 - gg + 2.0 * gg * rng.uniform());
                    double costheta = (1.0 + gg * gg - f * f) / (2.0 * gg);
                    kn = rotate_direction(kd, costheta, rng);
                }
                k = mk3((R)kn.x, (R)kn.y, (R)kn.z);
                nscatt++; c_scatt++;
                mode = M_MAIN1_START;
                break;
            }
            default: break;
            }
        }
        if (mode == M_DONE) break;

        // ---------------- one cell step of the current traversal
        int m; R ds;
        if (st.next(g, m, ds)) {
            c_steps++;
            double dtau = kappa_rho<R>(S, m, ell) * (double)ds;
            if (trav == T_PEEL) {
                tau += dtau;
            } else if (trav == T_MAIN1) {
                if (m >= 0) {
                    if (S.ncomp == 1) {
                        if (store) {
                            double Lintm = L * exp(-tau) * (-expm1(-dtau));
                            atomicAdd(labs + (size_t)m * nl + ell, (1.0 - S.albedo[ell]) * Lintm);
                            c_abs++;
                        }
                    } else {
                        double ksca = 0, kext = 0;
                        for (int h = 0; h < S.ncomp; h++) {
                            double rh = rho_load<R>(S, (size_t)h * S.ncells + m);
                            ksca += rh * S.ksca[h * nl + ell]; kext += rh * S.kext[h * nl + ell];
                        }
                        double alb = (kext > 0.0) ? ksca / kext : 0.0;
                        double Lintm = L * exp(-tau) * (-expm1(-dtau));
                        Lsca_acc += alb * Lintm;
                        if (store) { atomicAdd(labs + (size_t)m * nl + ell, (1.0 - alb) * Lintm); c_abs++; }
                    }
                }
                tau += dtau;
            } else {  // T_MAIN2
                double tn = tau + dtau, sn = s + (double)ds;
                if (tn > tau_int) {
                    s_int = s + ((tau_int - tau) / (tn - tau)) * (sn - s);
                    int_cell = m;
                    trav = T_NONE; mode = M_AFTER_MAIN2; c_trav++;
                    c_nbr += st.scanned; c_fb += st.fallbacks;
                } else { tau = tn; s = sn; }
            }
        } else {
            // traversal ended
            c_trav++;
            c_nbr += st.scanned; c_fb += st.fallbacks;
            if (st.steps > g.max_steps) { atomicOr(P.err, ERR_STEP_BUDGET); c_err++; }
            if (trav == T_PEEL) {
                detect_group(S, grp, ell, Lpeel, tau, scat_peel ? nscatt + 1 : 0, stellar,
                             (double)r.x, (double)r.y, (double)r.z, c_pix);
                c_peel++;
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

    atomicAdd(&s_cnt[0], (unsigned long long)c_pk);
    atomicAdd(&s_cnt[1], (unsigned long long)c_steps);
    atomicAdd(&s_cnt[2], (unsigned long long)c_trav);
    atomicAdd(&s_cnt[3], (unsigned long long)c_scatt);
    atomicAdd(&s_cnt[4], (unsigned long long)c_peel);
    atomicAdd(&s_cnt[5], (unsigned long long)c_abs);
    atomicAdd(&s_cnt[6], (unsigned long long)c_pix);
    atomicAdd(&s_cnt[7], (unsigned long long)c_nbr);
    atomicAdd(&s_cnt[8], (unsigned long long)c_fb);
    atomicAdd(&s_cnt[9], (unsigned long long)c_err);
    __syncthreads();
    if (threadIdx.x < 10) atomicAdd(P.counters + threadIdx.x, s_cnt[threadIdx.x]);
}

// ---------------------------------------------------------------------------------------------
template<typename R, template<typename> class Stepper>
static cudaError_t launch_one(const DevGrid& g, const DevScene* dS, const RunParams& P, int blocks,
                              int threads, cudaStream_t stream) {
    auto kern = tracer_kernel<R, Stepper>;
    if (blocks <= 0) {
        int dev = 0, sms = 0, per = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, threads, 0);
        blocks = sms * (per > 0 ? per : 1);
    }
    kern<<<blocks, threads, 0, stream>>>(g, dS, P);
    return cudaGetLastError();
}

cudaError_t launch_tracer(const DevGrid& g, const DevScene* dS, const RunParams& P, int precision,
                          int blocks, int threads, cudaStream_t stream) {
    if (threads <= 0) threads = 256;
    bool f64 = precision == SKG_PREC_FP64;
    switch (g.type) {
    case SKG_GRID_CARTESIAN:
        return f64 ? launch_one<double, CartStepper>(g, dS, P, blocks, threads, stream)
                   : launch_one<float, CartStepper>(g, dS, P, blocks, threads, stream);
    case SKG_GRID_OCTREE:
    case SKG_GRID_BINTREE:
        return f64 ? launch_one<double, TreeStepper>(g, dS, P, blocks, threads, stream)
                   : launch_one<float, TreeStepper>(g, dS, P, blocks, threads, stream);
    default:
        return f64 ? launch_one<double, VoronoiStepper>(g, dS, P, blocks, threads, stream)
                   : launch_one<float, VoronoiStepper>(g, dS, P, blocks, threads, stream);
    }
}

}  // namespace skg
