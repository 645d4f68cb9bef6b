// Thin C entry points around the reference's own geometry generator, compiled from the
// reference sources where they lie (see Makefile target `ref`). TEST INFRASTRUCTURE ONLY:
// used to pin the product's generator and to make the golden fixtures.
#include <cstdint>
#include <string>
#include "complab3d_geometry.hh"

extern "C" int ref_geom_generate(const char* kind, int nx, int ny, int nz, double porosity, double radius,
                                 double aperture, double roughness, int count, int layers,
                                 unsigned long long seed, const char* walls, int32_t* out_xfast) {
    complab_geom::GenOptions o;
    o.kind = kind; o.porosity = porosity; o.radius = radius; o.aperture = aperture;
    o.roughness = roughness; o.count = count; o.layers = layers; o.seed = seed; o.walls = walls;
    std::string err;
    complab_geom::Grid g = complab_geom::generate(nx, ny, nz, o, &err);
    if (g.size() == 0) return 1;
    for (size_t i = 0; i < g.size(); ++i) out_xfast[i] = g.v[i];
    return 0;
}

extern "C" int ref_geom_inspect(const int32_t* v_xfast, int nx, int ny, int nz, double* porosity,
                                long* open_voxels, long* isolated, int* clusters, int* spanning, int* percolates) {
    complab_geom::Grid g(nx, ny, nz);
    for (size_t i = 0; i < g.size(); ++i) g.v[i] = v_xfast[i];
    complab_geom::Inspection r = complab_geom::inspect(g);
    *porosity = r.porosity; *open_voxels = r.openVoxels; *isolated = r.isolatedVoxels;
    *clusters = r.clusters; *spanning = r.spanningClusters; *percolates = r.percolates ? 1 : 0;
    return 0;
}
