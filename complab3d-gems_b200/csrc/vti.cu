// vti.cu -- VTK ImageData (.vti) output of a domain's fields, as the reference's writers produce
// them (complab_functions.hh:96-176): the interior x-planes 1..nx-2 only (the inlet and outlet
// planes hold boundary values), x fastest in the file, spacing 1, one file per call.
//   writeNsVTI            -> CLB_FIELD_FLOW_VELOCITY: "velocityNorm" and "velocity" (float32)
//   writePorousMediumVTI  -> CLB_FIELD_MATERIAL: "tag" (float32 of the material codes)
//   writeAdvVTI           -> CLB_FIELD_CONCENTRATION / CLB_FIELD_BIOMASS: "Density" (float64)
// The XML is VTK's own format (version 1.0, UInt64 block headers, base64 binary data arrays),
// which ParaView reads. Host code only; the fields come through clb_get_field.
#include "clb_internal.cuh"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

using namespace clb;

namespace {

const char B64[] = "ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/";

void base64_append(std::string& out, const unsigned char* p, size_t n) {
    size_t i = 0;
    for (; i + 3 <= n; i += 3) {
        const uint32_t v = (uint32_t)p[i] << 16 | (uint32_t)p[i + 1] << 8 | p[i + 2];
        out += B64[v >> 18 & 63];
        out += B64[v >> 12 & 63];
        out += B64[v >> 6 & 63];
        out += B64[v & 63];
    }
    if (n - i == 1) {
        const uint32_t v = (uint32_t)p[i] << 16;
        out += B64[v >> 18 & 63];
        out += B64[v >> 12 & 63];
        out += "==";
    } else if (n - i == 2) {
        const uint32_t v = (uint32_t)p[i] << 16 | (uint32_t)p[i + 1] << 8;
        out += B64[v >> 18 & 63];
        out += B64[v >> 12 & 63];
        out += B64[v >> 6 & 63];
        out += '=';
    }
}

// One data array: the interior planes of a [components][N] field (x slowest), re-ordered to
// VTK's point order (x fastest) with the components of a point side by side, as `T`.
template <typename T, typename S>
std::string encode_array(const S* src, int comps, int nx, int ny, int nz) {
    const size_t N = (size_t)nx * ny * nz;
    const int ix = nx - 2;
    std::vector<T> buf((size_t)ix * ny * nz * comps);
    size_t o = 0;
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 1; x <= ix; ++x) {
                const size_t n = ((size_t)x * ny + y) * nz + z;
                for (int c = 0; c < comps; ++c) buf[o++] = (T)src[(size_t)c * N + n];
            }
    // base64 of the 8-byte block header (byte count) followed by base64 of the data, as VTK writes
    // a binary inline array with header_type UInt64
    const uint64_t bytes = (uint64_t)buf.size() * sizeof(T);
    std::string out;
    base64_append(out, reinterpret_cast<const unsigned char*>(&bytes), sizeof(bytes));
    base64_append(out, reinterpret_cast<const unsigned char*>(buf.data()), (size_t)bytes);
    return out;
}

}  // namespace

extern "C" {

clb_status clb_vti_write(const char* path, int nx, int ny, int nz, int n_arrays, const char* const* names,
                         const int32_t* components, const int32_t* dtypes, const void* const* data) {
    if (!path || (n_arrays > 0 && (!names || !components || !dtypes || !data)))
        return fail(nullptr, CLB_INVALID_ARG, "null argument");
    if (nx < 3 || ny < 1 || nz < 1) return fail(nullptr, CLB_INVALID_ARG, "domain too small for the interior planes");
    for (int a = 0; a < n_arrays; ++a) {
        if (!names[a] || !data[a]) return fail(nullptr, CLB_INVALID_ARG, "null array");
        if (components[a] < 1 || components[a] > 9) return fail(nullptr, CLB_INVALID_ARG, "1 to 9 components per array");
        if (dtypes[a] != 0 && dtypes[a] != 1) return fail(nullptr, CLB_INVALID_ARG, "arrays are float64 (0) or float32 (1)");
    }
    std::FILE* f = std::fopen(path, "wb");
    if (!f) return fail(nullptr, CLB_INVALID_ARG, std::string("cannot open ") + path);
    char ext[128];
    std::snprintf(ext, sizeof(ext), "0 %d 0 %d 0 %d", nx - 3, ny - 1, nz - 1);
    std::string s;
    s += "<?xml version=\"1.0\"?>\n";
    s += "<VTKFile type=\"ImageData\" version=\"1.0\" byte_order=\"LittleEndian\" header_type=\"UInt64\">\n";
    s += std::string("  <ImageData WholeExtent=\"") + ext + "\" Origin=\"0 0 0\" Spacing=\"1 1 1\">\n";
    s += std::string("    <Piece Extent=\"") + ext + "\">\n";
    s += "      <PointData>\n";
    for (int a = 0; a < n_arrays; ++a) {
        const bool f64 = dtypes[a] == 0;
        char head[256];
        std::snprintf(head, sizeof(head),
                      "        <DataArray type=\"%s\" Name=\"%s\" NumberOfComponents=\"%d\" format=\"binary\">\n",
                      f64 ? "Float64" : "Float32", names[a], components[a]);
        s += head;
        s += "          ";
        s += f64 ? encode_array<double>(static_cast<const double*>(data[a]), components[a], nx, ny, nz)
                 : encode_array<float>(static_cast<const float*>(data[a]), components[a], nx, ny, nz);
        s += "\n        </DataArray>\n";
    }
    s += "      </PointData>\n      <CellData>\n      </CellData>\n    </Piece>\n  </ImageData>\n</VTKFile>\n";
    const bool ok = std::fwrite(s.data(), 1, s.size(), f) == s.size();
    if (std::fclose(f) != 0 || !ok) return fail(nullptr, CLB_INVALID_ARG, std::string("cannot write ") + path);
    return CLB_OK;
}

clb_status clb_write_vti(clb_handle* h, int field, int index, const char* path) {
    if (!h || !path) return fail(h, CLB_INVALID_ARG, "null argument");
    const int nx = h->g.nx, ny = h->g.ny, nz = h->g.nz;
    const size_t N = (size_t)h->g.N;
    clb_status st;
    if (field == CLB_FIELD_FLOW_VELOCITY) {
        // computeVelocityNorm / computeVelocity in FP64, written as float32 (writeNsVTI)
        std::vector<double> u(3 * N);
        if ((st = clb_get_field(h, CLB_FIELD_FLOW_VELOCITY, 0, u.data(), 0)) != CLB_OK) return st;
        std::vector<float> norm(N), vel(3 * N);
        for (size_t n = 0; n < N; ++n) {
            const double a = u[n], b = u[N + n], c = u[2 * N + n];
            norm[n] = (float)std::sqrt(a * a + b * b + c * c);
            vel[n] = (float)a;
            vel[N + n] = (float)b;
            vel[2 * N + n] = (float)c;
        }
        const char* names[2] = {"velocityNorm", "velocity"};
        const int32_t comps[2] = {1, 3}, types[2] = {1, 1};
        const void* data[2] = {norm.data(), vel.data()};
        st = clb_vti_write(path, nx, ny, nz, 2, names, comps, types, data);
    } else if (field == CLB_FIELD_MATERIAL) {
        st = host_mat_sync(h);
        if (st != CLB_OK) return st;
        std::vector<float> tag(N);
        for (size_t n = 0; n < N; ++n) tag[n] = (float)h->h_mat[n];
        const char* names[1] = {"tag"};
        const int32_t comps[1] = {1}, types[1] = {1};
        const void* data[1] = {tag.data()};
        st = clb_vti_write(path, nx, ny, nz, 1, names, comps, types, data);
    } else if (field == CLB_FIELD_CONCENTRATION || field == CLB_FIELD_BIOMASS) {
        std::vector<double> c(N);
        if ((st = clb_get_field(h, field, index, c.data(), 0)) != CLB_OK) return st;
        const char* names[1] = {"Density"};
        const int32_t comps[1] = {1}, types[1] = {0};
        const void* data[1] = {c.data()};
        st = clb_vti_write(path, nx, ny, nz, 1, names, comps, types, data);
    } else {
        return fail(h, CLB_INVALID_ARG, "VTI output covers the flow velocity, the material map, concentrations and biomass");
    }
    if (st != CLB_OK) return fail(h, st, clb_global_error());
    return CLB_OK;
}

}  // extern "C"
