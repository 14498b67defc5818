// skg_setup.cu -- set-up kernels: cell density sampling, tree-node mass sampling, the dust
// emission spectra (equilibrium temperature + grey body) and the per-wavelength cell CDFs from
// which dust packets are launched.
#include "skg_scene.cuh"
#include "skg_internal.h"
#include <cub/device/device_scan.cuh>

namespace skg {

// DustSystem::setSampleDensityBody (DustSystem.cpp:145-172): the density of a cell is the average
// of Nrandom samples of sum_h norm_h rho_h(r) at random positions in the cell.  One thread per cell.
__global__ void sample_density_kernel(const DevGrid g, const DevGeometry* __restrict__ geoms,
                                      const double* __restrict__ norms, int ncomp, int ns, uint64_t seed,
                                      double* rho) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= g.ncells) return;
    Philox rng;
    rng.init(seed, (uint64_t)m, 0x00D5u);
    double sum[MAX_COMP] = {0, 0, 0, 0};
    for (int n = 0; n < ns; n++) {
        V3<double> p = random_position_in_cell(g, m, rng);
        for (int h = 0; h < ncomp; h++) sum[h] += norms[h] * geom_density(geoms[h], p.x, p.y, p.z);
    }
    for (int h = 0; h < ncomp; h++) rho[(size_t)h * g.ncells + m] = sum[h] / ns;
}

cudaError_t launch_sample_density(const DevGrid& g, const DevScene*, const void* dgeoms, const double* norms,
                                  int ncomp, int nsamples, uint64_t seed, double* rho, cudaStream_t s) {
    int th = 128;
    int bl = (g.ncells + th - 1) / th;
    if (bl == 0) return cudaSuccess;
    sample_density_kernel<<<bl, th, 0, s>>>(g, (const DevGeometry*)dgeoms, norms, ncomp, nsamples, seed, rho);
    return cudaGetLastError();
}

// TreeNodeSampleDensityCalculator (TreeNodeSampleDensityCalculator.cpp:26-80): Nrandom random
// positions in a node box; mass = mean density x volume, plus the min/max sample for the density
// dispersion criterion.  One warp per node, lanes split the samples.
__global__ void node_mass_kernel(const DevGeometry* __restrict__ geoms, const double* __restrict__ norms, int ncomp,
                                 const double* __restrict__ boxes, int nnodes, int ns, uint64_t seed,
                                 uint64_t node_offset, double* mass, double* rmin, double* rmax) {
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (warp >= nnodes) return;
    const double* b = boxes + 6 * (size_t)warp;
    double sum = 0, lo = DBL_MAX, hi = 0;
    for (int n = lane; n < ns; n += 32) {
        Philox rng;
        rng.init(seed, node_offset + warp, 0x7EE0000u + n);
        double x = rng.uniform(), y = rng.uniform(), z = rng.uniform();
        x = b[0] + x * (b[3] - b[0]); y = b[1] + y * (b[4] - b[1]); z = b[2] + z * (b[5] - b[2]);
        double rho = 0;
        for (int h = 0; h < ncomp; h++) rho += norms[h] * geom_density(geoms[h], x, y, z);
        sum += rho; lo = fmin(lo, rho); hi = fmax(hi, rho);
    }
    for (int o = 16; o > 0; o >>= 1) {
        sum += __shfl_down_sync(0xffffffffu, sum, o);
        lo = fmin(lo, __shfl_down_sync(0xffffffffu, lo, o));
        hi = fmax(hi, __shfl_down_sync(0xffffffffu, hi, o));
    }
    if (lane == 0) {
        double vol = (b[3] - b[0]) * (b[4] - b[1]) * (b[5] - b[2]);
        mass[warp] = sum / ns * vol;
        rmin[warp] = lo; rmax[warp] = hi;
    }
}

cudaError_t launch_node_mass(const void* dgeoms, const double* norms, int ncomp, const double* boxes,
                             int nnodes, int nsamples, uint64_t seed, uint64_t node_offset,
                             double* mass, double* rhomin, double* rhomax, cudaStream_t s) {
    if (nnodes <= 0) return cudaSuccess;
    int th = 256;
    int bl = (int)(((int64_t)nnodes * 32 + th - 1) / th);
    node_mass_kernel<<<bl, th, 0, s>>>((const DevGeometry*)dgeoms, norms, ncomp, boxes, nnodes, nsamples, seed,
                                       node_offset, mass, rhomin, rhomax);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------
// Dust emission spectra (one dust component, grey-body emissivity, every cell its own library
// entry: AllCellsDustLib + GreyBodyDustEmissivity).  Per cell:
//   J_ell = Labs(m,ell) / (kappa_abs rho 4 pi V) / dlambda            DustSystem.cpp:911-931
//   T     = invplanckabs( sum_ell kappa_abs J dlambda )                DustMix.cpp:674-697
//   L_ell = kappa_abs(ell) B_ell(T) dlambda, normalised to unit sum     GreyBodyDustEmissivity.cpp:21-45,
//                                                                       DustLib.cpp:135-148
// The mix's 1/mu factors cancel between the Planck table and the sum, as in the reference.
SKG_D double planck_B(double lambda, double T) {   // PlanckFunction.cpp:24-33
    const double h = 6.62606957e-34, c = 2.99792458e8, k = 1.3806488e-23;
    double x = h * c / (lambda * k * T);
    return 2.0 * h * c * c / pow(lambda, 5) / (exp(x) - 1.0);
}

SKG_D double cell_volume(const DevGrid& g, int m) {
    if (g.type == SKG_GRID_CARTESIAN) {
        int i = m / (g.nz * g.ny), j = (m / g.nz) % g.ny, k = m % g.nz;
        return (g.xv[i + 1] - g.xv[i]) * (g.yv[j + 1] - g.yv[j]) * (g.zv[k + 1] - g.zv[k]);
    } else if (g.type == SKG_GRID_VORONOI) {
        return g.vvol[m];
    }
    const double* b = g.node_box + 6 * (size_t)g.cell_node[m];
    return (b[3] - b[0]) * (b[4] - b[1]) * (b[5] - b[2]);
}

__global__ void dust_emission_kernel(const DevGrid g, const DevScene* __restrict__ Sp, const double* __restrict__ Tv,
                                     const double* __restrict__ planckabs, int nT, double* labsbol,
                                     double* spectra, double* temperature) {
    const DevScene& S = *Sp;
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= S.ncells) return;
    const int nl = S.nlambda;
    double lb = 0, pa = 0;
    double fac = 4.0 * M_PI * cell_volume(g, m);
    double rho = S.rho[m];
    for (int ell = 0; ell < nl; ell++) {
        double la = S.labs_stel[(size_t)ell * S.ncells + m] + S.labs_dust[(size_t)ell * S.ncells + m];
        lb += la;
        double kabs = S.kext[ell] * (1.0 - S.albedo[ell]);
        double J = la / (kabs * rho * fac) / S.dlambda[ell];
        if (!isfinite(J)) J = 0.0;
        pa += kabs * J * S.dlambda[ell];
    }
    labsbol[m] = lb;
    int p = dlocate_clip(planckabs, nT, pa);
    double T = Tv[p] + ((pa - planckabs[p]) / (planckabs[p + 1] - planckabs[p])) * (Tv[p + 1] - Tv[p]);
    if (temperature) temperature[m] = T;
    double total = 0;
    const size_t nc = (size_t)S.ncells;
    for (int ell = 0; ell < nl; ell++) {
        double kabs = S.kext[ell] * (1.0 - S.albedo[ell]);
        double v = (T > 0) ? kabs * planck_B(S.lambda[ell], T) * S.dlambda[ell] : 0.0;
        spectra[ell * nc + m] = v; total += v;
    }
    if (total > 0) for (int ell = 0; ell < nl; ell++) spectra[ell * nc + m] /= total;
}

cudaError_t launch_dust_emission(const DevGrid& g, const DevScene* dS, const double* Tv, const double* planckabs,
                                 int nT, double* labsbol, double* spectra, double* temperature, cudaStream_t s) {
    int th = 128;
    int bl = (g.ncells + th - 1) / th;
    if (bl == 0) return cudaSuccess;
    dust_emission_kernel<<<bl, th, 0, s>>>(g, dS, Tv, planckabs, nT, labsbol, spectra, temperature);
    return cudaGetLastError();
}

// emit_Lv[ell][m] = Labsbol[m] * spectrum[ell][m]   (PanMonteCarloSimulation.cpp:197-203)
__global__ void emission_weights_kernel(int nl, int nc, const double* __restrict__ labsbol,
                                        const double* __restrict__ spectra, double* emit_Lv) {
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)nl * nc) return;
    int ell = (int)(t / nc), m = (int)(t - (int64_t)ell * nc);
    double lb = labsbol[m];
    emit_Lv[t] = (lb > 0.0) ? lb * spectra[t] : 0.0;
}
// NR::cdf normalisation (NR.hpp:388-394): P_0 = 0, P_{i+1} = sum_{j<=i} p_j / sum p
__global__ void cdf_totals_kernel(int nl, int nc, double* cdf, double* Ltot) {
    int ell = blockIdx.x * blockDim.x + threadIdx.x;
    if (ell >= nl) return;
    Ltot[ell] = cdf[(size_t)ell * (nc + 1) + nc];
    cdf[(size_t)ell * (nc + 1)] = 0.0;
}
__global__ void cdf_normalise_kernel(int nl, int nc, double* cdf, const double* __restrict__ Ltot) {
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)nl * (nc + 1)) return;
    int ell = (int)(t / (nc + 1));
    double tot = Ltot[ell];
    if (t - (int64_t)ell * (nc + 1) == 0) return;
    cdf[t] = (tot > 0) ? cdf[t] / tot : 0.0;
}

size_t emission_scan_scratch_bytes(int ncells) {
    size_t bytes = 0;
    cub::DeviceScan::InclusiveSum(nullptr, bytes, (const double*)nullptr, (double*)nullptr, ncells);
    return bytes;
}

cudaError_t launch_emission_sources(const DevScene*, int nl, int nc, const double* labsbol, const double* spectra,
                                    double* emit_Lv, double* emit_cdf, double* emit_Ltot, void* scratch,
                                    size_t scratch_bytes, cudaStream_t s) {
    int64_t tot = (int64_t)nl * nc;
    emission_weights_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(nl, nc, labsbol, spectra, emit_Lv);
    for (int ell = 0; ell < nl; ell++) {
        size_t bytes = scratch_bytes;
        cudaError_t e = cub::DeviceScan::InclusiveSum(scratch, bytes, emit_Lv + (size_t)ell * nc,
                                                      emit_cdf + (size_t)ell * (nc + 1) + 1, nc, s);
        if (e != cudaSuccess) return e;
    }
    cdf_totals_kernel<<<(nl + 127) / 128, 128, 0, s>>>(nl, nc, emit_cdf, emit_Ltot);
    int64_t tc = (int64_t)nl * (nc + 1);
    cdf_normalise_kernel<<<(unsigned)((tc + 255) / 256), 256, 0, s>>>(nl, nc, emit_cdf, emit_Ltot);
    return cudaGetLastError();
}

// Writes each leaf's (single-component) density into its rope-tree record, so that a cell step
// of the FP32 walk reads box, density and ropes in one 64-byte gather.
__global__ void embed_density_kernel(float4* lrec, int nleaves, const float* __restrict__ rhof) {
    int li = blockIdx.x * blockDim.x + threadIdx.x;
    if (li >= nleaves) return;
    int cell = __float_as_int(lrec[4 * (size_t)li + 1].w);
    lrec[4 * (size_t)li].w = rhof[cell];
}
// The same for the lattice form: word 0 of cell m's 32-byte record.
__global__ void embed_density_lattice_kernel(uint4* prec, int ncells, const float* __restrict__ rhof) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= ncells) return;
    prec[2 * (size_t)m].x = __float_as_uint(rhof[m]);
}
cudaError_t launch_embed_density(const DevGrid& g, const float* rhof, cudaStream_t s) {
    int n = g.ncells;
    if (n <= 0) return cudaSuccess;
    if (g.lattice) embed_density_lattice_kernel<<<(n + 255) / 256, 256, 0, s>>>(const_cast<uint4*>(g.prec), n, rhof);
    else embed_density_kernel<<<(n + 255) / 256, 256, 0, s>>>(const_cast<float4*>(g.lrec), n, rhof);
    return cudaGetLastError();
}

// Sum of a vector (absorbed-luminosity totals for the self-absorption convergence test).
__global__ void sum_kernel(const double* __restrict__ x, int64_t n, double* out) {
    __shared__ double sh[256];
    double acc = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) acc += x[i];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) { if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o]; __syncthreads(); }
    if (threadIdx.x == 0) atomicAdd(out, sh[0]);
}
cudaError_t launch_sum(const double* x, int64_t n, double* out, cudaStream_t s) {
    cudaMemsetAsync(out, 0, sizeof(double), s);
    int bl = (int)std::min<int64_t>(1184, (n + 255) / 256);
    if (bl <= 0) return cudaSuccess;
    sum_kernel<<<bl, 256, 0, s>>>(x, n, out);
    return cudaGetLastError();
}

}  // namespace skg
