// skg_trace.cu -- per-ray DustGrid::path and Instrument::opticalDepth kernels.
//
// This translation unit is compiled with --fmad=false so that the FP64 steppers perform the
// reference's multiplies and adds as separately rounded operations (the reference's x86-64
// build has no FMA contraction), which makes cell sequences and segment lengths bit-identical
// to CartesianDustGrid::path, TreeDustGrid::path and VoronoiMesh::path.
#include "skg_scene.cuh"
#include "skg_internal.h"

namespace skg {

template<typename R, template<typename> class Stepper>
__global__ void count_segments_kernel(const DevGrid g, const double* __restrict__ r, const double* __restrict__ k,
                                      int64_t n, int64_t* counts, unsigned* err) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Stepper<R> st;
    st.init(g, (R)r[3 * i], (R)r[3 * i + 1], (R)r[3 * i + 2], (R)k[3 * i], (R)k[3 * i + 1], (R)k[3 * i + 2]);
    int m; R ds; int64_t c = 0;
    while (st.next(g, m, ds)) c++;
    if (st.steps > g.max_steps) atomicOr(err, ERR_STEP_BUDGET);
    counts[i] = c;
}

template<typename R, template<typename> class Stepper>
__global__ void write_segments_kernel(const DevGrid g, const double* __restrict__ r, const double* __restrict__ k,
                                      int64_t n, const int64_t* __restrict__ offsets, int32_t* cells,
                                      double* ds_out, unsigned* err) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Stepper<R> st;
    st.init(g, (R)r[3 * i], (R)r[3 * i + 1], (R)r[3 * i + 2], (R)k[3 * i], (R)k[3 * i + 1], (R)k[3 * i + 2]);
    int m; R ds;
    int64_t q = offsets[i], q1 = offsets[i + 1];
    while (st.next(g, m, ds)) {
        if (q >= q1) { atomicOr(err, ERR_CAPACITY); return; }
        cells[q] = m; ds_out[q] = (double)ds; q++;
    }
}

template<typename R> SKG_D double rho_at(const DevScene& S, size_t i);
template<> SKG_D double rho_at<double>(const DevScene& S, size_t i) { return S.rho[i]; }
template<> SKG_D double rho_at<float>(const DevScene& S, size_t i) { return (double)S.rhof[i]; }

// DustSystem::opticaldepth (DustSystem.cpp:960-976) with DustGridPath::opticalDepth (DustGridPath.hpp:97-108)
template<typename R, template<typename> class Stepper>
__global__ void optical_depth_kernel(const DevGrid g, const DevScene* __restrict__ Sp, const double* __restrict__ r,
                                     const double* __restrict__ k, int64_t n, int ell, double* tau_out, unsigned* err) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const DevScene& S = *Sp;
    Stepper<R> st;
    st.init(g, (R)r[3 * i], (R)r[3 * i + 1], (R)r[3 * i + 2], (R)k[3 * i], (R)k[3 * i + 1], (R)k[3 * i + 2]);
    int m; R ds;
    double tau = 0;
    while (st.next(g, m, ds)) {
        double kr = 0;
        if (m >= 0) for (int h = 0; h < S.ncomp; h++) kr += S.kext[h * S.nlambda + ell] * rho_at<R>(S, (size_t)h * S.ncells + m);
        tau += kr * (double)ds;
    }
    if (st.steps > g.max_steps) atomicOr(err, ERR_STEP_BUDGET);
    tau_out[i] = tau;
}

#define SKG_DISPATCH(KERNEL, ...)                                                                   \
    do {                                                                                            \
        int th = 128;                                                                               \
        int64_t bl = (n + th - 1) / th;                                                             \
        if (bl == 0) return cudaSuccess;                                                            \
        bool f64 = precision == SKG_PREC_FP64;                                                      \
        if (g.type == SKG_GRID_CARTESIAN) {                                                         \
            if (f64) KERNEL<double, CartStepper><<<bl, th, 0, s>>>(__VA_ARGS__);                    \
            else KERNEL<float, CartStepper><<<bl, th, 0, s>>>(__VA_ARGS__);                         \
        } else if (g.type == SKG_GRID_VORONOI) {                                                    \
            if (f64) KERNEL<double, VoronoiStepper><<<bl, th, 0, s>>>(__VA_ARGS__);                 \
            else KERNEL<float, VoronoiStepper><<<bl, th, 0, s>>>(__VA_ARGS__);                      \
        } else {                                                                                    \
            if (f64) KERNEL<double, TreeStepper><<<bl, th, 0, s>>>(__VA_ARGS__);                    \
            else if (g.search == SKG_SEARCH_BOOKKEEPING)                                            \
                KERNEL<float, TreeNodeWalk><<<bl, th, 0, s>>>(__VA_ARGS__);                         \
            else if (g.lattice)                                                                     \
                KERNEL<float, TreeLatticeStepper><<<bl, th, 0, s>>>(__VA_ARGS__);                   \
            else KERNEL<float, TreeStepper><<<bl, th, 0, s>>>(__VA_ARGS__);                         \
        }                                                                                           \
        return cudaGetLastError();                                                                  \
    } while (0)

cudaError_t launch_count_segments(const DevGrid& g, const double* r, const double* k, int64_t n,
                                  int precision, int64_t* counts, unsigned* err, cudaStream_t s) {
    SKG_DISPATCH(count_segments_kernel, g, r, k, n, counts, err);
}

cudaError_t launch_write_segments(const DevGrid& g, const double* r, const double* k, int64_t n,
                                  int precision, const int64_t* offsets, int32_t* cells, double* ds,
                                  unsigned* err, cudaStream_t s) {
    SKG_DISPATCH(write_segments_kernel, g, r, k, n, offsets, cells, ds, err);
}

cudaError_t launch_optical_depth(const DevGrid& g, const DevScene* dS, const double* r, const double* k,
                                 int64_t n, int ell, int precision, double* tau, unsigned* err,
                                 cudaStream_t s) {
    SKG_DISPATCH(optical_depth_kernel, g, dS, r, k, n, ell, tau, err);
}

}  // namespace skg
