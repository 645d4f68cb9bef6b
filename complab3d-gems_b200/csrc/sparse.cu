// sparse.cu -- host construction of the compacted node layout (see sparse.cuh).
#include "sparse.cuh"

#include <algorithm>
#include <cstring>

namespace clb {

void sparse_free(SparseBuffers& b) {
    cudaFree(b.node); cudaFree(b.code); cudaFree(b.wall); cudaFree(b.linkbase);
    cudaFree(b.rowstart); cudaFree(b.rowmask); cudaFree(b.rowpre); cudaFree(b.idx_of);
    b = SparseBuffers();
}

template <typename T>
static cudaError_t upload(T*& dst, const std::vector<T>& src, cudaStream_t s) {
    cudaError_t e = cudaMalloc(&dst, sizeof(T) * std::max<size_t>(1, src.size()));
    if (e != cudaSuccess || src.empty()) return e;
    return cudaMemcpyAsync(dst, src.data(), sizeof(T) * src.size(), cudaMemcpyHostToDevice, s);
}

clb_status sparse_build(clb_handle* h, const int8_t* stored_by_code, int q, SparseBuffers& out) {
    sparse_free(out);
    const Geom& G = h->g;
    const int nx = G.nx, ny = G.ny, nz = G.nz;
    const int64_t N = G.N;
    const int R = nx * ny, W = (nz + 31) / 32;
    std::vector<int32_t> idx(N, -1), node, rowstart(R), rowpre((size_t)R * W);
    std::vector<int8_t> code;
    std::vector<uint32_t> rowmask((size_t)R * W, 0u);
    node.reserve(N / 2);
    code.reserve(N / 2);
    int32_t K = 0;
    for (int r = 0; r < R; ++r) {
        rowstart[r] = K;
        int32_t pre = 0;
        for (int w = 0; w < W; ++w) {
            rowpre[(size_t)r * W + w] = pre;
            uint32_t m = 0;
            for (int b = 0; b < 32; ++b) {
                const int z = w * 32 + b;
                if (z >= nz) break;
                const int64_t n = (int64_t)r * nz + z;
                const int8_t c = h->h_mat[n];
                if (stored_by_code[(uint8_t)c & 127]) {
                    m |= 1u << b;
                    idx[n] = K++;
                    node.push_back((int32_t)n);
                    code.push_back(c);
                }
            }
            rowmask[(size_t)r * W + w] = m;
            pre += __builtin_popcount(m);
        }
    }
    std::vector<uint32_t> wall(K, 0u);
    std::vector<int32_t> linkbase(K, 0);
    int64_t L = 0;
    for (int32_t k = 0; k < K; ++k) {
        const int64_t n = node[k];
        const int x = (int)(n / G.plane), rr = (int)(n - (int64_t)x * G.plane), y = rr / nz, z = rr - y * nz;
        uint32_t wm = 0;
        for (int i = 1; i < q; ++i) {
            const int cx = q == 19 ? q19cx(i) : q7cx(i), cy = q == 19 ? q19cy(i) : q7cy(i),
                      cz = q == 19 ? q19cz(i) : q7cz(i);
            const int X = x + cx, Y = y + cy, Z = z + cz;
            if (X < 0 || Y < 0 || Z < 0 || X >= nx || Y >= ny || Z >= nz) continue;
            if (idx[(int64_t)X * G.plane + (int64_t)Y * nz + Z] < 0) wm |= 1u << i;
        }
        wall[k] = wm;
        linkbase[k] = (int32_t)L;
        L += __builtin_popcount(wm);
    }
    if (L > INT32_MAX) return fail(h, CLB_INVALID_ARG, "too many wall links");
    cudaError_t e = cudaSuccess;
    cudaStream_t s = h->stream;
    if (e == cudaSuccess) e = upload(out.node, node, s);
    if (e == cudaSuccess) e = upload(out.code, code, s);
    if (e == cudaSuccess) e = upload(out.wall, wall, s);
    if (e == cudaSuccess) e = upload(out.linkbase, linkbase, s);
    if (e == cudaSuccess) e = upload(out.rowstart, rowstart, s);
    if (e == cudaSuccess) e = upload(out.rowmask, rowmask, s);
    if (e == cudaSuccess) e = upload(out.rowpre, rowpre, s);
    if (e == cudaSuccess) e = upload(out.idx_of, idx, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // host vectors die here
    out.K = K;
    out.L = L;
    out.W = W;
    return cuda_check(h, e, "sparse layout");
}

}  // namespace clb
