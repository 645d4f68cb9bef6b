// geometry.cpp -- material maps on the host: the reference's generators, the .dat reader
// with ghost planes, the porosity-targeted sphere pack, and the percolation inspection.
//
// The generators must produce the reference's voxels for the same options
// (complab3d_geometry.hh:138-200), so they draw from the same xorshift64* stream
// (S. Vigna, "An experimental exploration of Marsaglia's xorshift generators, scrambled",
// 2016: shifts 12/25/27, multiplier 2685821657736338717, 53-bit uniform) in the same order and
// evaluate the same floating-point expressions in the same order. Results are returned in
// this library's layout (x slowest, z fastest); internally the grids are x fastest like the
// reference's.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/clb.h"

namespace clb {
clb_status fail(clb_handle* h, clb_status s, const std::string& msg);
}

namespace {

const int G_SOLID = 0, G_WALL = 1, G_PORE = 2;

struct XorShift64Star {
    uint64_t s;
    explicit XorShift64Star(uint64_t seed) : s(seed ? seed : 1) {}
    uint64_t next() {
        s ^= s >> 12;
        s ^= s << 25;
        s ^= s >> 27;
        return s * 2685821657736338717ULL;
    }
    double uniform() { return (double)(next() >> 11) / 9007199254740992.0; }
    int below(int n) { return n > 0 ? (int)(uniform() * (double)n) : 0; }
};

// x-fastest working grid
struct Vol {
    int nx, ny, nz;
    std::vector<int> v;
    Vol(int a, int b, int c, int fill) : nx(a), ny(b), nz(c), v((size_t)a * b * c, fill) {}
    size_t at(int x, int y, int z) const { return (size_t)x + (size_t)nx * ((size_t)y + (size_t)ny * (size_t)z); }
};

void add_walls(Vol& g, const std::string& axes) {
    const bool all = axes == "all";
    const bool wx = all || axes.find('x') != std::string::npos;
    const bool wy = all || axes.find('y') != std::string::npos;
    const bool wz = all || axes.find('z') != std::string::npos;
    for (int z = 0; z < g.nz; ++z)
        for (int y = 0; y < g.ny; ++y)
            for (int x = 0; x < g.nx; ++x) {
                const bool ox = x == 0 || x == g.nx - 1, oy = y == 0 || y == g.ny - 1, oz = z == 0 || z == g.nz - 1;
                if ((wx && ox) || (wy && oy) || (wz && oz)) g.v[g.at(x, y, z)] = G_WALL;
            }
}

// 27-point periodic box average, terms summed dz, dy, dx outermost to innermost.
void box_smooth(std::vector<double>& f, int nx, int ny, int nz, int passes) {
    std::vector<double> t(f.size());
    for (int p = 0; p < passes; ++p) {
        for (int z = 0; z < nz; ++z)
            for (int y = 0; y < ny; ++y)
                for (int x = 0; x < nx; ++x) {
                    double s = 0.0;
                    int cnt = 0;
                    for (int dz = -1; dz <= 1; ++dz)
                        for (int dy = -1; dy <= 1; ++dy)
                            for (int dx = -1; dx <= 1; ++dx) {
                                const int X = (x + dx + nx) % nx, Y = (y + dy + ny) % ny, Z = (z + dz + nz) % nz;
                                s += f[(size_t)X + (size_t)nx * ((size_t)Y + (size_t)ny * (size_t)Z)];
                                ++cnt;
                            }
                    t[(size_t)x + (size_t)nx * ((size_t)y + (size_t)ny * (size_t)z)] = s / (double)cnt;
                }
        f.swap(t);
    }
}

void to_library_layout(const Vol& g, int8_t* out) {
    for (int x = 0; x < g.nx; ++x)
        for (int y = 0; y < g.ny; ++y)
            for (int z = 0; z < g.nz; ++z) out[((size_t)x * g.ny + y) * g.nz + z] = (int8_t)g.v[g.at(x, y, z)];
}

}  // namespace

extern "C" {

clb_status clb_geom_generate(const clb_geom_options* o, int nx, int ny, int nz, int8_t* out) {
    if (!o || !out || !o->kind) return clb::fail(nullptr, CLB_INVALID_ARG, "null argument");
    if (nx < 1 || ny < 1 || nz < 1) return clb::fail(nullptr, CLB_INVALID_ARG, "bad size");
    const std::string kind = o->kind;
    const std::string walls = o->walls ? o->walls : "";
    Vol g(nx, ny, nz, G_PORE);
    XorShift64Star rng(o->seed);
    if (kind == "channel") {
    } else if (kind == "spheres" || kind == "cylinders") {
        const bool cyl = kind == "cylinders";
        for (int k = 0; k < o->count; ++k) {
            const int cx = rng.below(nx);
            const int cy = rng.below(ny);
            const int cz = cyl ? 0 : rng.below(nz);
            const double r2 = o->radius * o->radius;
            for (int z = 0; z < nz; ++z)
                for (int y = 0; y < ny; ++y)
                    for (int x = 0; x < nx; ++x) {
                        const double dx = x - cx, dy = y - cy, dz = cyl ? 0.0 : (double)(z - cz);
                        if (dx * dx + dy * dy + dz * dz <= r2) g.v[g.at(x, y, z)] = G_SOLID;
                    }
        }
    } else if (kind == "random") {
        std::vector<double> f(g.v.size());
        for (size_t i = 0; i < f.size(); ++i) f[i] = rng.uniform();
        box_smooth(f, nx, ny, nz, 2);
        std::vector<double> sorted(f);
        std::sort(sorted.begin(), sorted.end());
        const size_t cut = (size_t)((1.0 - o->porosity) * (double)sorted.size());
        const double thr = sorted[cut < sorted.size() ? cut : sorted.size() - 1];
        for (size_t i = 0; i < f.size(); ++i) g.v[i] = (f[i] >= thr) ? G_PORE : G_SOLID;
    } else if (kind == "fracture") {
        std::fill(g.v.begin(), g.v.end(), G_SOLID);
        const double mid = 0.5 * ny;
        for (int z = 0; z < nz; ++z) {
            std::vector<double> wob((size_t)nx, 0.0);
            for (int k = 1; k <= 3; ++k) {
                const double ph = rng.uniform() * 6.283185307179586;
                for (int x = 0; x < nx; ++x)
                    wob[(size_t)x] += (o->roughness / k) * std::sin(6.283185307179586 * k * x / nx + ph);
            }
            for (int x = 0; x < nx; ++x)
                for (int y = 0; y < ny; ++y)
                    if (std::fabs(y - (mid + wob[(size_t)x])) <= 0.5 * o->aperture) g.v[g.at(x, y, z)] = G_PORE;
        }
    } else if (kind == "layered") {
        for (int i = 0; i < o->layers; ++i) {
            const int y0 = (int)((double)i * ny / o->layers);
            const int y1 = (int)((double)(i + 1) * ny / o->layers);
            const double p = o->porosity * ((i % 2 == 0) ? 1.4 : 0.5);
            const double pc = p < 1.0 ? p : 1.0;
            for (int z = 0; z < nz; ++z)
                for (int y = y0; y < y1; ++y)
                    for (int x = 0; x < nx; ++x)
                        if (rng.uniform() > pc) g.v[g.at(x, y, z)] = G_SOLID;
        }
    } else {
        return clb::fail(nullptr, CLB_INVALID_ARG, "unknown geometry kind '" + kind + "'");
    }
    if (walls != "none" && !walls.empty()) add_walls(g, walls);
    to_library_layout(g, out);
    return CLB_OK;
}

clb_status clb_geom_sphere_pack(int nx, int ny, int nz, double porosity, double rmin, double rmax, uint64_t seed,
                                const char* walls, int grain, int wall, int pore, int8_t* out) {
    if (!out || nx < 1 || ny < 1 || nz < 1) return clb::fail(nullptr, CLB_INVALID_ARG, "bad arguments");
    if (!(porosity > 0 && porosity < 1) || !(rmin > 0) || rmax < rmin)
        return clb::fail(nullptr, CLB_INVALID_ARG, "bad porosity or radius range");
    const size_t N = (size_t)nx * ny * nz;
    std::vector<int8_t> m(N, (int8_t)pore);
    auto id = [&](int x, int y, int z) { return ((size_t)x * ny + y) * nz + z; };
    const std::string w = walls ? walls : "";
    const bool all = w == "all";
    const bool wx = all || w.find('x') != std::string::npos;
    const bool wy = all || w.find('y') != std::string::npos;
    const bool wz = all || w.find('z') != std::string::npos;
    size_t open = N;
    for (int x = 0; x < nx; ++x)
        for (int y = 0; y < ny; ++y)
            for (int z = 0; z < nz; ++z) {
                const bool ox = x == 0 || x == nx - 1, oy = y == 0 || y == ny - 1, oz = z == 0 || z == nz - 1;
                if ((wx && ox) || (wy && oy) || (wz && oz)) { m[id(x, y, z)] = (int8_t)wall; --open; }
            }
    XorShift64Star rng(seed);
    const size_t target = (size_t)(porosity * (double)N);
    int guard = 0;
    while (open > target && guard < 10000000) {
        ++guard;
        const int cx = rng.below(nx), cy = rng.below(ny), cz = rng.below(nz);
        const double r = rmin + (rmax - rmin) * rng.uniform();
        const int ri = (int)std::ceil(r);
        const double r2 = r * r;
        for (int x = std::max(0, cx - ri); x <= std::min(nx - 1, cx + ri); ++x)
            for (int y = std::max(0, cy - ri); y <= std::min(ny - 1, cy + ri); ++y)
                for (int z = std::max(0, cz - ri); z <= std::min(nz - 1, cz + ri); ++z) {
                    const double dx = x - cx, dy = y - cy, dz = z - cz;
                    if (dx * dx + dy * dy + dz * dz > r2) continue;
                    int8_t& v = m[id(x, y, z)];
                    if (v == (int8_t)pore) { v = (int8_t)grain; --open; }
                }
    }
    std::memcpy(out, m.data(), N);
    return CLB_OK;
}

clb_status clb_geom_read_dat(const char* path, int nx_inner, int ny, int nz, int8_t* out) {
    if (!path || !out || nx_inner < 1 || ny < 1 || nz < 1) return clb::fail(nullptr, CLB_INVALID_ARG, "bad arguments");
    FILE* fp = std::fopen(path, "r");
    if (!fp) return clb::fail(nullptr, CLB_INVALID_ARG, std::string("cannot open ") + path);
    const size_t P = (size_t)ny * nz;
    std::vector<int8_t> slice(P);
    for (int x = 1; x <= nx_inner; ++x) {
        for (size_t p = 0; p < P; ++p) {
            long v;
            if (std::fscanf(fp, "%ld", &v) != 1) {
                std::fclose(fp);
                return clb::fail(nullptr, CLB_INVALID_ARG, "geometry file ends early");
            }
            if (v < 0 || v > 127) {
                std::fclose(fp);
                return clb::fail(nullptr, CLB_INVALID_ARG, "material code outside 0..127");
            }
            slice[p] = (int8_t)v;
        }
        std::memcpy(out + (size_t)x * P, slice.data(), P);
        if (x == 1) std::memcpy(out, slice.data(), P);
        if (x == nx_inner) std::memcpy(out + (size_t)(nx_inner + 1) * P, slice.data(), P);
    }
    std::fclose(fp);
    return CLB_OK;
}

clb_status clb_geom_inspect(const int8_t* map, int nx, int ny, int nz, clb_inspection* out) {
    if (!map || !out || nx < 1 || ny < 1 || nz < 1) return clb::fail(nullptr, CLB_INVALID_ARG, "bad arguments");
    const size_t N = (size_t)nx * ny * nz;
    auto id = [&](int x, int y, int z) { return ((size_t)x * ny + y) * nz + z; };
    std::vector<char> open(N, 0);
    int64_t nopen = 0;
    for (size_t i = 0; i < N; ++i)
        if (map[i] >= G_PORE) { open[i] = 1; ++nopen; }
    std::vector<int> lab(N, 0);
    int cur = 0;
    std::vector<size_t> stack;
    const int dx[6] = {1, -1, 0, 0, 0, 0}, dy[6] = {0, 0, 1, -1, 0, 0}, dz[6] = {0, 0, 0, 0, 1, -1};
    for (size_t s = 0; s < N; ++s) {
        if (!open[s] || lab[s]) continue;
        ++cur;
        stack.clear();
        stack.push_back(s);
        lab[s] = cur;
        while (!stack.empty()) {
            const size_t i = stack.back();
            stack.pop_back();
            const int x = (int)(i / ((size_t)ny * nz));
            const int y = (int)((i / (size_t)nz) % (size_t)ny);
            const int z = (int)(i % (size_t)nz);
            for (int d = 0; d < 6; ++d) {
                const int X = x + dx[d], Y = y + dy[d], Z = z + dz[d];
                if (X < 0 || Y < 0 || Z < 0 || X >= nx || Y >= ny || Z >= nz) continue;
                const size_t j = id(X, Y, Z);
                if (open[j] && !lab[j]) { lab[j] = cur; stack.push_back(j); }
            }
        }
    }
    std::vector<char> at_in((size_t)cur + 1, 0), at_out((size_t)cur + 1, 0), span((size_t)cur + 1, 0);
    for (int y = 0; y < ny; ++y)
        for (int z = 0; z < nz; ++z) {
            if (lab[id(0, y, z)]) at_in[(size_t)lab[id(0, y, z)]] = 1;
            if (lab[id(nx - 1, y, z)]) at_out[(size_t)lab[id(nx - 1, y, z)]] = 1;
        }
    int nspan = 0;
    for (int c = 1; c <= cur; ++c)
        if (at_in[(size_t)c] && at_out[(size_t)c]) { span[(size_t)c] = 1; ++nspan; }
    int64_t iso = 0;
    for (size_t i = 0; i < N; ++i)
        if (open[i] && !span[(size_t)lab[i]]) ++iso;
    int q2 = 1;
    for (int x = 0; x < nx && q2; ++x)
        for (int y = 0; y < ny && q2; ++y)
            for (int z = 1; z < nz; ++z)
                if (map[id(x, y, z)] != map[id(x, y, 0)]) { q2 = 0; break; }
    out->porosity = (double)nopen / (double)N;
    out->open_voxels = nopen;
    out->isolated_voxels = iso;
    out->clusters = cur;
    out->spanning_clusters = nspan;
    out->percolates = nspan > 0;
    out->quasi_2d = q2;
    return CLB_OK;
}

}  // extern "C"
