// skg_voronoi.cu -- Voronoi tessellation of the dust grid sites (VoronoiMesh::buildMesh).
#include "skg_scene.cuh"
#include "skg_internal.h"

using namespace skg;

struct skg_voronoi {
    int n = 0;
};

extern "C" {

int skg_voronoi_build(const double*, int32_t, double, double, double, double, double, double, int, skg_voronoi** out) {
    *out = nullptr;
    set_error("Voronoi construction is not available in this build");
    return SKG_ERR_INVALID;
}
int skg_voronoi_sizes(const skg_voronoi*, int32_t*, int64_t*, int32_t*, int64_t*) { return SKG_ERR_INVALID; }
int skg_voronoi_arrays(const skg_voronoi*, int64_t*, int32_t*, double*, double*, double*, int64_t*, int32_t*) {
    return SKG_ERR_INVALID;
}
int skg_voronoi_grid(const skg_voronoi*, skg_grid*) { return SKG_ERR_INVALID; }
int skg_voronoi_destroy(skg_voronoi* v) { delete v; return SKG_OK; }

}  // extern "C"
