// skg_internal.h -- declarations shared between the library's translation units.
#pragma once
#include "../../include/skirt_b200.h"
#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>

namespace skg {

struct DevGrid;
struct DevScene;
struct RunParams;

// skg_trace.cu (compiled with --fmad=false: bit-exact FP64 traversal)
cudaError_t launch_count_segments(const DevGrid& g, const double* r, const double* k, int64_t n,
                                  int precision, int64_t* counts, unsigned* err, cudaStream_t s);
cudaError_t launch_write_segments(const DevGrid& g, const double* r, const double* k, int64_t n,
                                  int precision, const int64_t* offsets, int32_t* cells, double* ds,
                                  unsigned* err, cudaStream_t s);
cudaError_t launch_optical_depth(const DevGrid& g, const DevScene* dS, const double* r, const double* k,
                                 int64_t n, int ell, int precision, double* tau, unsigned* err,
                                 cudaStream_t s);

// skg_setup.cu
cudaError_t launch_sample_density(const DevGrid& g, const DevScene* dS, const void* dgeoms,
                                  const double* norms, int ncomp, int nsamples, uint64_t seed,
                                  double* rho, cudaStream_t s);
cudaError_t launch_node_mass(const void* dgeoms, const double* norms, int ncomp, const double* boxes,
                             int nnodes, int nsamples, uint64_t seed, uint64_t node_offset,
                             double* mass, double* rhomin, double* rhomax, cudaStream_t s);
cudaError_t launch_dust_emission(const DevGrid& g, const DevScene* dS, const double* Tv,
                                 const double* planckabs, int nT, double* labsbol, double* spectra,
                                 double* temperature, cudaStream_t s);
cudaError_t launch_emission_sources(const DevScene* dS, int nlambda, int ncells, const double* labsbol,
                                    const double* spectra, double* emit_Lv, double* emit_cdf,
                                    double* emit_Ltot, void* scratch, size_t scratch_bytes,
                                    cudaStream_t s);
size_t emission_scan_scratch_bytes(int ncells);
cudaError_t launch_sum(const double* x, int64_t n, double* out, cudaStream_t s);
cudaError_t launch_embed_density(const DevGrid& g, const float* rhof, cudaStream_t s);

// skg_host.cpp
void sersic_table(double n, double* sv, double* Sv, double* Mv);      // 101 points each
void chunk_params(double packages, int nthreads, int nprocs, int nlambda,
                  uint64_t& nchunks, uint64_t& chunksize, uint64_t& npp);

// error message of the calling thread
void set_error(const std::string& msg);
const char* get_error();

}  // namespace skg
